// ============================================================================
// pxr_oracle.cpp -- CPU oracle for the PICSAR per-step particle loop.
//
// TEST INFRASTRUCTURE ONLY.  This file restates, routine by routine, the
// reference Fortran 90 hot path of PICSAR (ECP-WarpX/picsar, src/...) in
// C++17 so that the B200 CUDA kernels can be checked against it.  Only the
// tests, the smoke check and the CPU-baseline leg of the benchmark load it;
// no product code path links, imports or calls it.
//
// Parity status: PINNED.  The reference ships no golden vectors and its
// Fortran cannot be compiled in this image (no Fortran compiler), so the
// reference's own routines are translated statement by statement to C
// (oracle/ftrans.py: same types, loop bounds, operation order and intrinsic
// semantics) and every kernel restated here is checked bit for bit against
// them (tests/test_oracle_vs_reference.py): pushers, fused gather+push 1-3,
// scalar gathers, Esirkepov 1-3 and _n, charge deposition, Yee.  The
// reference's cross-variant checks and physics invariants are reproduced on
// top (tests/test_oracle_cpu.py).
//
// Array convention: every grid is a Fortran column-major array with lower
// bound -g and upper bound n+g per axis (x fastest), passed as a base pointer
// to element (-gx,-gy,-gz).  Units: constants clight, mu0, eps0 are inputs so
// both the SI build and the LIBRARY build (c = mu0 = eps0 = 1,
// src/modules/modules.F90:62-73) are expressible.
// Build: oracle/Makefile (g++ -O3 -fopenmp -ffp-contract=off).
// ============================================================================
#include <cmath>
#include <cstdint>
#include <cstring>
#include <cstdlib>
#include <vector>
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef int64_t i64;

namespace {

// Fortran array view with arbitrary lower bounds (column-major).
struct F3 {
  double* p;
  i64 lo0, lo1, lo2;
  i64 n0, n1;  // extents of the first two axes
  inline double& operator()(i64 i, i64 j, i64 k) const {
    return p[(i - lo0) + n0 * ((j - lo1) + n1 * (k - lo2))];
  }
};

// (-g:n+g) per axis
inline F3 gview(double* p, i64 nx, i64 ny, i64 nz, i64 gx, i64 gy, i64 gz) {
  (void)nz;
  F3 a;
  a.p = p; a.lo0 = -gx; a.lo1 = -gy; a.lo2 = -gz;
  a.n0 = nx + 1 + 2 * gx; a.n1 = ny + 1 + 2 * gy;
  return a;
}

// (lo:hi) per axis
inline F3 bview(double* p, const i64* lo, const i64* hi) {
  F3 a;
  a.p = p; a.lo0 = lo[0]; a.lo1 = lo[1]; a.lo2 = lo[2];
  a.n0 = hi[0] - lo[0] + 1; a.n1 = hi[1] - lo[1] + 1;
  return a;
}

inline i64 ffloor(double x) { return (i64)std::floor(x); }
// Fortran NINT: nearest integer, halves rounded away from zero.
inline i64 fnint(double x) { return (i64)std::lround(x); }
inline double sq(double x) { return x * x; }

const double onesixth = 1.0 / 6.0;
const double twothird = 2.0 / 3.0;

}  // namespace

extern "C" {

// ----------------------------------------------------------------------------
// Pushers.  src/particle_pushers/boris_pusher/boris_3d.F90:51-141 (Boris u),
// :849-893 (pushxyz), :1059-1107 (set_gamma); vay_pusher/vay_3d.F90:56-139.
// ----------------------------------------------------------------------------
void orc_boris_push_u_3d(i64 np, double* uxp, double* uyp, double* uzp,
                         double* gaminv, const double* ex, const double* ey,
                         const double* ez, const double* bx, const double* by,
                         const double* bz, double q, double m, double dt,
                         double clight) {
  const double cst = q * dt * 0.5 / m;
  const double clghtisq = 1.0 / sq(clight);
  for (i64 ip = 0; ip < np; ++ip) {
    uxp[ip] = uxp[ip] + ex[ip] * cst;
    uyp[ip] = uyp[ip] + ey[ip] * cst;
    uzp[ip] = uzp[ip] + ez[ip] * cst;
    double usq = (sq(uxp[ip]) + sq(uyp[ip]) + sq(uzp[ip])) * clghtisq;
    double gaminvtmp = 1.0 / std::sqrt(1.0 + usq);
    double tx = gaminvtmp * bx[ip] * cst;
    double ty = gaminvtmp * by[ip] * cst;
    double tz = gaminvtmp * bz[ip] * cst;
    double tsqi = 2.0 / (1.0 + sq(tx) + sq(ty) + sq(tz));
    double sx = tx * tsqi, sy = ty * tsqi, sz = tz * tsqi;
    double uxppr = uxp[ip] + uyp[ip] * tz - uzp[ip] * ty;
    double uyppr = uyp[ip] + uzp[ip] * tx - uxp[ip] * tz;
    double uzppr = uzp[ip] + uxp[ip] * ty - uyp[ip] * tx;
    uxp[ip] = uxp[ip] + uyppr * sz - uzppr * sy;
    uyp[ip] = uyp[ip] + uzppr * sx - uxppr * sz;
    uzp[ip] = uzp[ip] + uxppr * sy - uyppr * sx;
    uxp[ip] = uxp[ip] + ex[ip] * cst;
    uyp[ip] = uyp[ip] + ey[ip] * cst;
    uzp[ip] = uzp[ip] + ez[ip] * cst;
    usq = (sq(uxp[ip]) + sq(uyp[ip]) + sq(uzp[ip])) * clghtisq;
    gaminv[ip] = 1.0 / std::sqrt(1.0 + usq);
  }
}

void orc_set_gamma(i64 np, const double* uxp, const double* uyp,
                   const double* uzp, double* gaminv, double clight) {
  const double clghtisq = 1.0 / sq(clight);
  for (i64 ip = 0; ip < np; ++ip) {
    double usq = (sq(uxp[ip]) + sq(uyp[ip]) + sq(uzp[ip])) * clghtisq;
    gaminv[ip] = 1.0 / std::sqrt(1.0 + usq);
  }
}

void orc_pushxyz(i64 np, double* xp, double* yp, double* zp, const double* uxp,
                 const double* uyp, const double* uzp, const double* gaminv,
                 double dt) {
  for (i64 ip = 0; ip < np; ++ip) {
    xp[ip] = xp[ip] + uxp[ip] * gaminv[ip] * dt;
    yp[ip] = yp[ip] + uyp[ip] * gaminv[ip] * dt;
    zp[ip] = zp[ip] + uzp[ip] * gaminv[ip] * dt;
  }
}

void orc_ebcancelpush3d(i64 np, double* uxp, double* uyp, double* uzp,
                        double* gi, const double* ex, const double* ey,
                        const double* ez, const double* bx, const double* by,
                        const double* bz, double q, double m, double dt,
                        i64 which, double clight) {
  const double invclight = 1.0 / clight;
  const double invclightsq = 1.0 / (clight * clight);
  if (which == 0) {
    const double cst = q * dt / m;
    const double bconst = 0.5 * cst;
    for (i64 ip = 0; ip < np; ++ip) {
      double taux = bconst * bx[ip], tauy = bconst * by[ip], tauz = bconst * bz[ip];
      double tausq = taux * taux + tauy * tauy + tauz * tauz;
      double uxpr = uxp[ip] + cst * ex[ip] + (uyp[ip] * tauz - uzp[ip] * tauy) * gi[ip];
      double uypr = uyp[ip] + cst * ey[ip] + (uzp[ip] * taux - uxp[ip] * tauz) * gi[ip];
      double uzpr = uzp[ip] + cst * ez[ip] + (uxp[ip] * tauy - uyp[ip] * taux) * gi[ip];
      double gprsq = (1.0 + (uxpr * uxpr + uypr * uypr + uzpr * uzpr) * invclightsq);
      double ust = (uxpr * taux + uypr * tauy + uzpr * tauz) * invclight;
      double sigma = gprsq - tausq;
      double gisq = 2.0 / (sigma + std::sqrt(sigma * sigma + 4.0 * (tausq + ust * ust)));
      gi[ip] = std::sqrt(gisq);
      double bg = bconst * gi[ip];
      double tx = bg * bx[ip], ty = bg * by[ip], tz = bg * bz[ip];
      double s = 1.0 / (1.0 + tausq * gisq);
      double tu = tx * uxpr + ty * uypr + tz * uzpr;
      uxp[ip] = s * (uxpr + tx * tu + uypr * tz - uzpr * ty);
      uyp[ip] = s * (uypr + ty * tu + uzpr * tx - uxpr * tz);
      uzp[ip] = s * (uzpr + tz * tu + uxpr * ty - uypr * tx);
    }
  } else if (which == 1) {
    const double cst = 0.5 * q * dt / m;
    for (i64 ip = 0; ip < np; ++ip) {
      double vx = uxp[ip] * gi[ip], vy = uyp[ip] * gi[ip], vz = uzp[ip] * gi[ip];
      uxp[ip] = uxp[ip] + cst * (ex[ip] + vy * bz[ip] - vz * by[ip]);
      uyp[ip] = uyp[ip] + cst * (ey[ip] + vz * bx[ip] - vx * bz[ip]);
      uzp[ip] = uzp[ip] + cst * (ez[ip] + vx * by[ip] - vy * bx[ip]);
      gi[ip] = 1.0 / std::sqrt(1.0 + (uxp[ip] * uxp[ip] + uyp[ip] * uyp[ip] +
                                      uzp[ip] * uzp[ip]) * invclightsq);
    }
  } else if (which == 2) {
    const double cst = 0.5 * q * dt / m;
    const double bconst = cst;
    for (i64 ip = 0; ip < np; ++ip) {
      double uxpr = uxp[ip] + cst * ex[ip];
      double uypr = uyp[ip] + cst * ey[ip];
      double uzpr = uzp[ip] + cst * ez[ip];
      double gprsq = (1.0 + (uxpr * uxpr + uypr * uypr + uzpr * uzpr) * invclightsq);
      double taux = bconst * bx[ip], tauy = bconst * by[ip], tauz = bconst * bz[ip];
      double tausq = taux * taux + tauy * tauy + tauz * tauz;
      double ust = (uxpr * taux + uypr * tauy + uzpr * tauz) * invclight;
      double sigma = gprsq - tausq;
      double gisq = 2.0 / (sigma + std::sqrt(sigma * sigma + 4.0 * (tausq + ust * ust)));
      gi[ip] = std::sqrt(gisq);
      double bg = bconst * gi[ip];
      double tx = bg * bx[ip], ty = bg * by[ip], tz = bg * bz[ip];
      double s = 1.0 / (1.0 + tausq * gisq);
      double tu = tx * uxpr + ty * uypr + tz * uzpr;
      uxp[ip] = s * (uxpr + tx * tu + uypr * tz - uzpr * ty);
      uyp[ip] = s * (uypr + ty * tu + uzpr * tx - uxpr * tz);
      uzp[ip] = s * (uzpr + tz * tu + uxpr * ty - uypr * tx);
    }
  }
}

// ----------------------------------------------------------------------------
// Fused energy-conserving gather + push, l_lower_order_in_v = .TRUE. only
// (the fused kernels implement only that branch).
// src/particle_pushers/particle_pusher_manager_3d.F90:1287-1482 (order 1),
// :1522-1818 (order 2), :1820-2193 (order 3).  The gather accumulates (+=)
// into ex..bz; the pusher and pushxyz use the module time step `dt`
// (the argument dtt only enters const1, which the kernels never use).
// particle_pusher: 0 = Boris + set_gamma, 1 = Vay (which=0).
// ----------------------------------------------------------------------------
static void push_block(i64 pusher, i64 n, double* ux, double* uy, double* uz,
                       double* gi, double* ex, double* ey, double* ez,
                       double* bx, double* by, double* bz, double* x, double* y,
                       double* z, double q, double m, double dt, double clight) {
  if (pusher == 1) {
    orc_ebcancelpush3d(n, ux, uy, uz, gi, ex, ey, ez, bx, by, bz, q, m, dt, 0, clight);
  } else {
    orc_boris_push_u_3d(n, ux, uy, uz, gi, ex, ey, ez, bx, by, bz, q, m, dt, clight);
    orc_set_gamma(n, ux, uy, uz, gi, clight);
  }
  orc_pushxyz(n, x, y, z, ux, uy, uz, gi, dt);
}

void orc_field_gathering_plus_particle_pusher_1_1_1(
    i64 np, double* xp, double* yp, double* zp, double* uxp, double* uyp,
    double* uzp, double* gaminv, double* ex, double* ey, double* ez, double* bx,
    double* by, double* bz, double xmin, double ymin, double zmin, double dx,
    double dy, double dz, i64 nx, i64 ny, i64 nz, i64 nxguard, i64 nyguard,
    i64 nzguard, double* exg_, double* eyg_, double* ezg_, double* bxg_,
    double* byg_, double* bzg_, double q, double m, i64 lvect, double dt,
    i64 pusher, double clight) {
  F3 exg = gview(exg_, nx, ny, nz, nxguard, nyguard, nzguard);
  F3 eyg = gview(eyg_, nx, ny, nz, nxguard, nyguard, nzguard);
  F3 ezg = gview(ezg_, nx, ny, nz, nxguard, nyguard, nzguard);
  F3 bxg = gview(bxg_, nx, ny, nz, nxguard, nyguard, nzguard);
  F3 byg = gview(byg_, nx, ny, nz, nxguard, nyguard, nzguard);
  F3 bzg = gview(bzg_, nx, ny, nz, nxguard, nyguard, nzguard);
  const double dxi = 1.0 / dx, dyi = 1.0 / dy, dzi = 1.0 / dz;
  double sx[2], sy[2], sz[2];
  for (i64 ip = 0; ip < np; ip += lvect) {
    i64 bs = std::min(lvect, np - ip);
    for (i64 nn = ip; nn < ip + bs; ++nn) {
      double x = (xp[nn] - xmin) * dxi;
      double y = (yp[nn] - ymin) * dyi;
      double z = (zp[nn] - zmin) * dzi;
      i64 j = ffloor(x), j0 = ffloor(x);
      i64 k = ffloor(y), k0 = ffloor(y);
      i64 l = ffloor(z), l0 = ffloor(z);
      double xint = x - j, yint = y - k, zint = z - l;
      sx[0] = 1.0 - xint; sx[1] = xint;
      sy[0] = 1.0 - yint; sy[1] = yint;
      sz[0] = 1.0 - zint; sz[1] = zint;
      double a;
      a = (sy[0] * exg(j0, k, l) + sy[1] * exg(j0, k + 1, l)) * sz[0] +
          (sy[0] * exg(j0, k, l + 1) + sy[1] * exg(j0, k + 1, l + 1)) * sz[1];
      ex[nn] = ex[nn] + a;
      a = (sx[0] * eyg(j, k0, l) + sx[1] * eyg(j + 1, k0, l)) * sz[0] +
          (sx[0] * eyg(j, k0, l + 1) + sx[1] * eyg(j + 1, k0, l + 1)) * sz[1];
      ey[nn] = ey[nn] + a;
      a = (sx[0] * ezg(j, k, l0) + sx[1] * ezg(j + 1, k, l0)) * sy[0] +
          (sx[0] * ezg(j, k + 1, l0) + sx[1] * ezg(j + 1, k + 1, l0)) * sy[1];
      ez[nn] = ez[nn] + a;
      a = (sx[0] * bxg(j, k0, l0) + sx[1] * bxg(j + 1, k0, l0));
      bx[nn] = bx[nn] + a;
      a = (sy[0] * byg(j0, k, l0) + sy[1] * byg(j0, k + 1, l0));
      by[nn] = by[nn] + a;
      a = (sz[0] * bzg(j0, k0, l) + sz[1] * bzg(j0, k0, l + 1));
      bz[nn] = bz[nn] + a;
    }
    push_block(pusher, bs, uxp + ip, uyp + ip, uzp + ip, gaminv + ip, ex + ip,
               ey + ip, ez + ip, bx + ip, by + ip, bz + ip, xp + ip, yp + ip,
               zp + ip, q, m, dt, clight);
  }
}

void orc_field_gathering_plus_particle_pusher_2_2_2(
    i64 np, double* xp, double* yp, double* zp, double* uxp, double* uyp,
    double* uzp, double* gaminv, double* ex, double* ey, double* ez, double* bx,
    double* by, double* bz, double xmin, double ymin, double zmin, double dx,
    double dy, double dz, i64 nx, i64 ny, i64 nz, i64 nxguard, i64 nyguard,
    i64 nzguard, double* exg_, double* eyg_, double* ezg_, double* bxg_,
    double* byg_, double* bzg_, double q, double m, i64 lvect, double dt,
    i64 pusher, double clight) {
  F3 exg = gview(exg_, nx, ny, nz, nxguard, nyguard, nzguard);
  F3 eyg = gview(eyg_, nx, ny, nz, nxguard, nyguard, nzguard);
  F3 ezg = gview(ezg_, nx, ny, nz, nxguard, nyguard, nzguard);
  F3 bxg = gview(bxg_, nx, ny, nz, nxguard, nyguard, nzguard);
  F3 byg = gview(byg_, nx, ny, nz, nxguard, nyguard, nzguard);
  F3 bzg = gview(bzg_, nx, ny, nz, nxguard, nyguard, nzguard);
  const double dxi = 1.0 / dx, dyi = 1.0 / dy, dzi = 1.0 / dz;
  // arrays (-1:1) stored at offset +1
  double sx_[3], sy_[3], sz_[3], sx0_[3], sy0_[3], sz0_[3];
  double *sx = sx_ + 1, *sy = sy_ + 1, *sz = sz_ + 1;
  double *sx0 = sx0_ + 1, *sy0 = sy0_ + 1, *sz0 = sz0_ + 1;
  for (int t = 0; t < 3; ++t) sx_[t] = sy_[t] = sz_[t] = sx0_[t] = sy0_[t] = sz0_[t] = 0.0;
  for (i64 ip = 0; ip < np; ip += lvect) {
    i64 bs = std::min(lvect, np - ip);
    for (i64 nn = ip; nn < ip + bs; ++nn) {
      double x = (xp[nn] - xmin) * dxi;
      double y = (yp[nn] - ymin) * dyi;
      double z = (zp[nn] - zmin) * dzi;
      i64 j = fnint(x), j0 = ffloor(x - 0.5);
      i64 k = fnint(y), k0 = ffloor(y - 0.5);
      i64 l = fnint(z), l0 = ffloor(z - 0.5);
      double xint = x - j, yint = y - k, zint = z - l;
      double xintsq = xint * xint;
      sx[-1] = 0.5 * sq(0.5 - xint); sx[0] = 0.75 - xintsq; sx[1] = 0.5 * sq(0.5 + xint);
      double yintsq = yint * yint;
      sy[-1] = 0.5 * sq(0.5 - yint); sy[0] = 0.75 - yintsq; sy[1] = 0.5 * sq(0.5 + yint);
      double zintsq = zint * zint;
      sz[-1] = 0.5 * sq(0.5 - zint); sz[0] = 0.75 - zintsq; sz[1] = 0.5 * sq(0.5 + zint);
      xint = x - 0.5 - j0; yint = y - 0.5 - k0; zint = z - 0.5 - l0;
      sx0[0] = 1.0 - xint; sx0[1] = xint;
      sy0[0] = 1.0 - yint; sy0[1] = yint;
      sz0[0] = 1.0 - zint; sz0[1] = zint;
      double a;
      // Ex: x staggered (linear at j0), y,z quadratic at k,l
      for (int ll = -1; ll <= 1; ++ll) {
        a = (sx0[0] * exg(j0, k - 1, l + ll) + sx0[1] * exg(j0 + 1, k - 1, l + ll)) * sy[-1];
        a = a + (sx0[0] * exg(j0, k, l + ll) + sx0[1] * exg(j0 + 1, k, l + ll)) * sy[0];
        a = a + (sx0[0] * exg(j0, k + 1, l + ll) + sx0[1] * exg(j0 + 1, k + 1, l + ll)) * sy[1];
        ex[nn] = ex[nn] + a * sz[ll];
      }
      // Ey
      for (int ll = -1; ll <= 1; ++ll) {
        a = (sx[-1] * eyg(j - 1, k0, l + ll) + sx[0] * eyg(j, k0, l + ll) +
             sx[1] * eyg(j + 1, k0, l + ll)) * sy0[0];
        a = a + (sx[-1] * eyg(j - 1, k0 + 1, l + ll) + sx[0] * eyg(j, k0 + 1, l + ll) +
                 sx[1] * eyg(j + 1, k0 + 1, l + ll)) * sy0[1];
        ey[nn] = ey[nn] + a * sz[ll];
      }
      // Ez
      for (int ll = 0; ll <= 1; ++ll) {
        a = (sx[-1] * ezg(j - 1, k - 1, l0 + ll) + sx[0] * ezg(j, k - 1, l0 + ll) +
             sx[1] * ezg(j + 1, k - 1, l0 + ll)) * sy[-1];
        a = a + (sx[-1] * ezg(j - 1, k, l0 + ll) + sx[0] * ezg(j, k, l0 + ll) +
                 sx[1] * ezg(j + 1, k, l0 + ll)) * sy[0];
        a = a + (sx[-1] * ezg(j - 1, k + 1, l0 + ll) + sx[0] * ezg(j, k + 1, l0 + ll) +
                 sx[1] * ezg(j + 1, k + 1, l0 + ll)) * sy[1];
        ez[nn] = ez[nn] + a * sz0[ll];
      }
      // Bx
      for (int ll = 0; ll <= 1; ++ll) {
        a = (sx[-1] * bxg(j - 1, k0, l0 + ll) + sx[0] * bxg(j, k0, l0 + ll) +
             sx[1] * bxg(j + 1, k0, l0 + ll)) * sy0[0];
        a = a + (sx[-1] * bxg(j - 1, k0 + 1, l0 + ll) + sx[0] * bxg(j, k0 + 1, l0 + ll) +
                 sx[1] * bxg(j + 1, k0 + 1, l0 + ll)) * sy0[1];
        bx[nn] = bx[nn] + a * sz0[ll];
      }
      // By
      for (int ll = 0; ll <= 1; ++ll) {
        a = (sx0[0] * byg(j0, k - 1, l0 + ll) + sx0[1] * byg(j0 + 1, k - 1, l0 + ll)) * sy[-1];
        a = a + (sx0[0] * byg(j0, k, l0 + ll) + sx0[1] * byg(j0 + 1, k, l0 + ll)) * sy[0];
        a = a + (sx0[0] * byg(j0, k + 1, l0 + ll) + sx0[1] * byg(j0 + 1, k + 1, l0 + ll)) * sy[1];
        by[nn] = by[nn] + a * sz0[ll];
      }
      // Bz
      for (int ll = -1; ll <= 1; ++ll) {
        a = (sx0[0] * bzg(j0, k0, l + ll) + sx0[1] * bzg(j0 + 1, k0, l + ll)) * sy0[0];
        a = a + (sx0[0] * bzg(j0, k0 + 1, l + ll) + sx0[1] * bzg(j0 + 1, k0 + 1, l + ll)) * sy0[1];
        bz[nn] = bz[nn] + a * sz[ll];
      }
    }
    push_block(pusher, bs, uxp + ip, uyp + ip, uzp + ip, gaminv + ip, ex + ip,
               ey + ip, ez + ip, bx + ip, by + ip, bz + ip, xp + ip, yp + ip,
               zp + ip, q, m, dt, clight);
  }
}

void orc_field_gathering_plus_particle_pusher_3_3_3(
    i64 np, double* xp, double* yp, double* zp, double* uxp, double* uyp,
    double* uzp, double* gaminv, double* ex, double* ey, double* ez, double* bx,
    double* by, double* bz, double xmin, double ymin, double zmin, double dx,
    double dy, double dz, i64 nx, i64 ny, i64 nz, i64 nxguard, i64 nyguard,
    i64 nzguard, double* exg_, double* eyg_, double* ezg_, double* bxg_,
    double* byg_, double* bzg_, double q, double m, i64 lvect, double dt,
    i64 pusher, double clight) {
  F3 exg = gview(exg_, nx, ny, nz, nxguard, nyguard, nzguard);
  F3 eyg = gview(eyg_, nx, ny, nz, nxguard, nyguard, nzguard);
  F3 ezg = gview(ezg_, nx, ny, nz, nxguard, nyguard, nzguard);
  F3 bxg = gview(bxg_, nx, ny, nz, nxguard, nyguard, nzguard);
  F3 byg = gview(byg_, nx, ny, nz, nxguard, nyguard, nzguard);
  F3 bzg = gview(bzg_, nx, ny, nz, nxguard, nyguard, nzguard);
  const double dxi = 1.0 / dx, dyi = 1.0 / dy, dzi = 1.0 / dz;
  double sx_[4], sy_[4], sz_[4], sx0_[3], sy0_[3], sz0_[3];
  double *sx = sx_ + 1, *sy = sy_ + 1, *sz = sz_ + 1;     // (-1:2)
  double *sx0 = sx0_ + 1, *sy0 = sy0_ + 1, *sz0 = sz0_ + 1;  // (-1:1)
  for (i64 ip = 0; ip < np; ip += lvect) {
    i64 bs = std::min(lvect, np - ip);
    for (i64 nn = ip; nn < ip + bs; ++nn) {
      double x = (xp[nn] - xmin) * dxi;
      double y = (yp[nn] - ymin) * dyi;
      double z = (zp[nn] - zmin) * dzi;
      i64 j = ffloor(x), j0 = ffloor(x);
      i64 k = ffloor(y), k0 = ffloor(y);
      i64 l = ffloor(z), l0 = ffloor(z);
      double xint = x - j, yint = y - k, zint = z - l;
      double oxint = 1.0 - xint, xintsq = xint * xint, oxintsq = oxint * oxint;
      sx[-1] = onesixth * oxintsq * oxint;
      sx[0] = twothird - xintsq * (1.0 - xint * 0.5);
      sx[1] = twothird - oxintsq * (1.0 - oxint * 0.5);
      sx[2] = onesixth * xintsq * xint;
      double oyint = 1.0 - yint, yintsq = yint * yint, oyintsq = oyint * oyint;
      sy[-1] = onesixth * oyintsq * oyint;
      sy[0] = twothird - yintsq * (1.0 - yint * 0.5);
      sy[1] = twothird - oyintsq * (1.0 - oyint * 0.5);
      sy[2] = onesixth * yintsq * yint;
      double ozint = 1.0 - zint, zintsq = zint * zint, ozintsq = ozint * ozint;
      sz[-1] = onesixth * ozintsq * ozint;
      sz[0] = twothird - zintsq * (1.0 - zint * 0.5);
      sz[1] = twothird - ozintsq * (1.0 - ozint * 0.5);
      sz[2] = onesixth * zintsq * zint;
      xint = x - 0.5 - j0; yint = y - 0.5 - k0; zint = z - 0.5 - l0;
      xintsq = xint * xint;
      sx0[-1] = 0.5 * sq(0.5 - xint); sx0[0] = 0.75 - xintsq; sx0[1] = 0.5 * sq(0.5 + xint);
      yintsq = yint * yint;
      sy0[-1] = 0.5 * sq(0.5 - yint); sy0[0] = 0.75 - yintsq; sy0[1] = 0.5 * sq(0.5 + yint);
      zintsq = zint * zint;
      sz0[-1] = 0.5 * sq(0.5 - zint); sz0[0] = 0.75 - zintsq; sz0[1] = 0.5 * sq(0.5 + zint);
      double a;
      // Ex: x quadratic-staggered at j0 (-1:1), y,z cubic at k,l (-1:2)
      for (int ll = -1; ll <= 2; ++ll) {
        a = (sx0[-1] * exg(j0 - 1, k - 1, l + ll) + sx0[0] * exg(j0, k - 1, l + ll) +
             sx0[1] * exg(j0 + 1, k - 1, l + ll)) * sy[-1];
        for (int kk = 0; kk <= 2; ++kk)
          a = a + (sx0[-1] * exg(j0 - 1, k + kk, l + ll) + sx0[0] * exg(j0, k + kk, l + ll) +
                   sx0[1] * exg(j0 + 1, k + kk, l + ll)) * sy[kk];
        ex[nn] = ex[nn] + a * sz[ll];
      }
      // Ey: x cubic, y staggered, z cubic
      for (int ll = -1; ll <= 2; ++ll) {
        a = (sx[-1] * eyg(j - 1, k0 - 1, l + ll) + sx[0] * eyg(j, k0 - 1, l + ll) +
             sx[1] * eyg(j + 1, k0 - 1, l + ll) + sx[2] * eyg(j + 2, k0 - 1, l + ll)) * sy0[-1];
        for (int kk = 0; kk <= 1; ++kk)
          a = a + (sx[-1] * eyg(j - 1, k0 + kk, l + ll) + sx[0] * eyg(j, k0 + kk, l + ll) +
                   sx[1] * eyg(j + 1, k0 + kk, l + ll) + sx[2] * eyg(j + 2, k0 + kk, l + ll)) *
                      sy0[kk];
        ey[nn] = ey[nn] + a * sz[ll];
      }
      // Ez: x cubic, y cubic, z staggered
      for (int ll = -1; ll <= 1; ++ll) {
        a = (sx[-1] * ezg(j - 1, k - 1, l0 + ll) + sx[0] * ezg(j, k - 1, l0 + ll) +
             sx[1] * ezg(j + 1, k - 1, l0 + ll) + sx[2] * ezg(j + 2, k - 1, l0 + ll)) * sy[-1];
        for (int kk = 0; kk <= 2; ++kk)
          a = a + (sx[-1] * ezg(j - 1, k + kk, l0 + ll) + sx[0] * ezg(j, k + kk, l0 + ll) +
                   sx[1] * ezg(j + 1, k + kk, l0 + ll) + sx[2] * ezg(j + 2, k + kk, l0 + ll)) *
                      sy[kk];
        ez[nn] = ez[nn] + a * sz0[ll];
      }
      // Bx: x cubic, y staggered, z staggered
      for (int ll = -1; ll <= 1; ++ll) {
        a = (sx[-1] * bxg(j - 1, k0 - 1, l0 + ll) + sx[0] * bxg(j, k0 - 1, l0 + ll) +
             sx[1] * bxg(j + 1, k0 - 1, l0 + ll) + sx[2] * bxg(j + 2, k0 - 1, l0 + ll)) * sy0[-1];
        for (int kk = 0; kk <= 1; ++kk)
          a = a + (sx[-1] * bxg(j - 1, k0 + kk, l0 + ll) + sx[0] * bxg(j, k0 + kk, l0 + ll) +
                   sx[1] * bxg(j + 1, k0 + kk, l0 + ll) + sx[2] * bxg(j + 2, k0 + kk, l0 + ll)) *
                      sy0[kk];
        bx[nn] = bx[nn] + a * sz0[ll];
      }
      // By: x staggered, y cubic, z staggered
      for (int ll = -1; ll <= 1; ++ll) {
        a = (sx0[-1] * byg(j0 - 1, k - 1, l0 + ll) + sx0[0] * byg(j0, k - 1, l0 + ll) +
             sx0[1] * byg(j0 + 1, k - 1, l0 + ll)) * sy[-1];
        for (int kk = 0; kk <= 2; ++kk)
          a = a + (sx0[-1] * byg(j0 - 1, k + kk, l0 + ll) + sx0[0] * byg(j0, k + kk, l0 + ll) +
                   sx0[1] * byg(j0 + 1, k + kk, l0 + ll)) * sy[kk];
        by[nn] = by[nn] + a * sz0[ll];
      }
      // Bz: x staggered, y staggered, z cubic
      for (int ll = -1; ll <= 2; ++ll) {
        a = (sx0[-1] * bzg(j0 - 1, k0 - 1, l + ll) + sx0[0] * bzg(j0, k0 - 1, l + ll) +
             sx0[1] * bzg(j0 + 1, k0 - 1, l + ll)) * sy0[-1];
        for (int kk = 0; kk <= 1; ++kk)
          a = a + (sx0[-1] * bzg(j0 - 1, k0 + kk, l + ll) + sx0[0] * bzg(j0, k0 + kk, l + ll) +
                   sx0[1] * bzg(j0 + 1, k0 + kk, l + ll)) * sy0[kk];
        bz[nn] = bz[nn] + a * sz[ll];
      }
    }
    push_block(pusher, bs, uxp + ip, uyp + ip, uzp + ip, gaminv + ip, ex + ip,
               ey + ip, ez + ip, bx + ip, by + ip, bz + ip, xp + ip, yp + ip,
               zp + ip, q, m, dt, clight);
  }
}

// pxr_particle_bin_sorting (src/housekeeping/sorting.F90:247-361) on one set
// of flat arrays: bin id iz*nx3*ny3 + iy*nx3 + ix + 1 from floor((x - xmin2) *
// dxi), counts per bin, exclusive prefix, then each particle in input order
// to the next slot of its bin; the weight column w (may be NULL) travels with
// the particles.  Bins outside the range (a DEBUG-only STOP in the reference)
// are clamped to the nearest end bin.
void orc_particle_bin_sorting(i64 np2, double* xp, double* yp, double* zp, double* ux,
                              double* uy, double* uz, double* gam, double* w, double xmin2,
                              double ymin2, double zmin2, double xmax2, double ymax2,
                              double zmax2, double dxf, double dyf, double dzf) {
  const double dxi = 1. / dxf, dyi = 1. / dyf, dzi = 1. / dzf;
  const i64 nx3 = (i64)std::ceil((xmax2 - xmin2) * dxi);
  const i64 ny3 = (i64)std::ceil((ymax2 - ymin2) * dyi);
  const i64 nz3 = (i64)std::ceil((zmax2 - zmin2) * dzi);
  const i64 nbhc = nx3 * ny3 * nz3;
  std::vector<i64> hcnb(np2), piihc(nbhc + 1, 0), nbppc(nbhc + 1, 0);
  for (i64 ip = 0; ip < np2; ++ip) {
    const double x2 = (xp[ip] - xmin2) * dxi, y2 = (yp[ip] - ymin2) * dyi,
                 z2 = (zp[ip] - zmin2) * dzi;
    const i64 ix = ffloor(x2), iy = ffloor(y2), iz = ffloor(z2);
    i64 h = iz * nx3 * ny3 + iy * nx3 + ix + 1;
    h = h < 1 ? 1 : (h > nbhc ? nbhc : h);
    hcnb[ip] = h;
    nbppc[h] = nbppc[h] + 1;
  }
  i64 k = 0;
  for (i64 ic = 1; ic <= nbhc; ++ic) {
    piihc[ic] = k;
    k = k + nbppc[ic];
  }
  std::vector<i64> dest(np2);
  for (i64 ip = 0; ip < np2; ++ip) {
    const i64 kk = hcnb[ip];
    piihc[kk] = piihc[kk] + 1;
    dest[ip] = piihc[kk] - 1;              // 1-based slot piihc(k) -> 0-based
  }
  double* cols[8] = {xp, yp, zp, ux, uy, uz, gam, w};
  std::vector<double> tmp(np2);
  for (double* c : cols) {
    if (!c) continue;
    for (i64 ip = 0; ip < np2; ++ip) tmp[dest[ip]] = c[ip];
    std::copy(tmp.begin(), tmp.end(), c);
  }
}

}  // extern "C"

// ----------------------------------------------------------------------------
// Scalar energy-conserving gathers, both l_lower_order_in_v branches and the
// nodal-grid switch.  Restates gete3d/getb3d_energy_conserving_scalar_{1,2,3}:
// src/field_gathering/energy_conserving/field_gathering_o1_3d.F90:74-580,
// _o2_3d.F90:70-620, _o3_3d.F90:83-660.  Each component is summed as
//   f(ip) += s_x(jj)*s_y(kk)*s_z(ll)*g(...)  over (ll, kk, jj) loops.
// Node-centred axes use the full-order shape at j = floor(x) (odd order) or
// nint(x) (even order); the staggered axis uses either the order-1 lower
// shape (l_lower_order_in_v) or the full order, at the index the Fortran
// computes from stagger_shift = 0.5 (0 when l_nodal).
// ----------------------------------------------------------------------------
namespace {
struct Shape {
  i64 i0;         // base index
  int lo, hi;     // inclusive offset range
  double s[5];    // s[off - lo]
};

// Full-order shape of a node-centred axis.
inline void node_shape(int order, double x, Shape& sh) {
  if (order == 1) {
    sh.i0 = ffloor(x); double xi = x - sh.i0;
    sh.lo = 0; sh.hi = 1; sh.s[0] = 1.0 - xi; sh.s[1] = xi;
  } else if (order == 2) {
    sh.i0 = fnint(x); double xi = x - sh.i0, xs = xi * xi;
    sh.lo = -1; sh.hi = 1;
    sh.s[0] = 0.5 * sq(0.5 - xi); sh.s[1] = 0.75 - xs; sh.s[2] = 0.5 * sq(0.5 + xi);
  } else {
    sh.i0 = ffloor(x); double xi = x - sh.i0;
    double ox = 1.0 - xi, xs = xi * xi, oxs = ox * ox;
    sh.lo = -1; sh.hi = 2;
    sh.s[0] = onesixth * oxs * ox;
    sh.s[1] = twothird - xs * (1.0 - xi * 0.5);
    sh.s[2] = twothird - oxs * (1.0 - ox * 0.5);
    sh.s[3] = onesixth * xs * xi;
  }
}

// Staggered-axis shape (index and interpolation variable as in the scalar
// Fortran routines).
inline void stag_shape(int order, bool lower, double ss, double x, Shape& sh) {
  if (order == 1) {
    if (lower) {
      sh.i0 = ffloor(x + 0.5 - ss); sh.lo = 0; sh.hi = 0; sh.s[0] = 1.0;
    } else {
      sh.i0 = ffloor(x - ss); double xi = x - ss - sh.i0;
      sh.lo = 0; sh.hi = 1; sh.s[0] = 1.0 - xi; sh.s[1] = xi;
    }
  } else if (order == 2) {
    if (lower) {
      sh.i0 = ffloor(x - ss); double xi = x - ss - sh.i0;
      sh.lo = 0; sh.hi = 1; sh.s[0] = 1.0 - xi; sh.s[1] = xi;
    } else {
      sh.i0 = ffloor(x + 0.5 - ss); double xi = x - ss - sh.i0, xs = xi * xi;
      sh.lo = -1; sh.hi = 1;
      sh.s[0] = 0.5 * sq(0.5 - xi); sh.s[1] = 0.75 - xs; sh.s[2] = 0.5 * sq(0.5 + xi);
    }
  } else {
    if (lower) {
      sh.i0 = ffloor(x + 0.5 - ss); double xi = x - ss - sh.i0, xs = xi * xi;
      sh.lo = -1; sh.hi = 1;
      sh.s[0] = 0.5 * sq(0.5 - xi); sh.s[1] = 0.75 - xs; sh.s[2] = 0.5 * sq(0.5 + xi);
    } else {
      sh.i0 = ffloor(x - ss); double xi = x - ss - sh.i0;
      double ox = 1.0 - xi, xs = xi * xi, oxs = ox * ox;
      sh.lo = -1; sh.hi = 2;
      sh.s[0] = onesixth * oxs * ox;
      sh.s[1] = twothird - xs * (1.0 - xi * 0.5);
      sh.s[2] = twothird - oxs * (1.0 - ox * 0.5);
      sh.s[3] = onesixth * xs * xi;
    }
  }
}

inline double gather3(const F3& g, const Shape& a, const Shape& b, const Shape& c,
                      double acc) {
  for (int ll = c.lo; ll <= c.hi; ++ll)
    for (int kk = b.lo; kk <= b.hi; ++kk)
      for (int jj = a.lo; jj <= a.hi; ++jj)
        acc = acc + a.s[jj - a.lo] * b.s[kk - b.lo] * c.s[ll - c.lo] *
                        g(a.i0 + jj, b.i0 + kk, c.i0 + ll);
  return acc;
}
}  // namespace

extern "C" {

// which: 0 = E (gete3d), 1 = B (getb3d).  Accumulates into f1,f2,f3.
void orc_geteb3d_energy_conserving_scalar(
    i64 which, i64 np, const double* xp, const double* yp, const double* zp,
    double* f1, double* f2, double* f3, double xmin, double ymin, double zmin,
    double dx, double dy, double dz, i64 nx, i64 ny, i64 nz, i64 nxguard,
    i64 nyguard, i64 nzguard, i64 order, double* g1_, double* g2_, double* g3_,
    i64 l_lower_order_in_v, i64 l_nodal) {
  F3 g1 = gview(g1_, nx, ny, nz, nxguard, nyguard, nzguard);
  F3 g2 = gview(g2_, nx, ny, nz, nxguard, nyguard, nzguard);
  F3 g3 = gview(g3_, nx, ny, nz, nxguard, nyguard, nzguard);
  const double ss = l_nodal ? 0.0 : 0.5;
  const bool lower = l_lower_order_in_v != 0;
  const double dxi = 1.0 / dx, dyi = 1.0 / dy, dzi = 1.0 / dz;
  for (i64 ip = 0; ip < np; ++ip) {
    double x = (xp[ip] - xmin) * dxi, y = (yp[ip] - ymin) * dyi, z = (zp[ip] - zmin) * dzi;
    Shape nxs, nys, nzs, sxs, sys, szs;
    node_shape((int)order, x, nxs); node_shape((int)order, y, nys); node_shape((int)order, z, nzs);
    stag_shape((int)order, lower, ss, x, sxs);
    stag_shape((int)order, lower, ss, y, sys);
    stag_shape((int)order, lower, ss, z, szs);
    if (which == 0) {
      f1[ip] = gather3(g1, sxs, nys, nzs, f1[ip]);
      f2[ip] = gather3(g2, nxs, sys, nzs, f2[ip]);
      f3[ip] = gather3(g3, nxs, nys, szs, f3[ip]);
    } else {
      f1[ip] = gather3(g1, nxs, sys, szs, f1[ip]);
      f2[ip] = gather3(g2, sxs, nys, szs, f2[ip]);
      f3[ip] = gather3(g3, sxs, sys, nzs, f3[ip]);
    }
  }
}

// ----------------------------------------------------------------------------
// 2D (x-z) path.  Grids are 2-D Fortran arrays (-g:n+g) in x and z.
// Gathers: pxr_gete2dxz / pxr_getb2dxz_energy_conserving_scalar_{1_1,2_2,3_3}
// (src/field_gathering/energy_conserving/field_gathering_o{1,2,3}_2d.F90),
// the 3-D scalar forms without the y axis: components summed as
//   f(ip) += s_x(jj)*s_z(ll)*g(...) over (ll, jj).
// E: Ex (stag x, node z), Ey (node, node), Ez (node x, stag z); B: Bx (node
// x, stag z), By (stag, stag), Bz (stag x, node z).
// ----------------------------------------------------------------------------
struct F2 {
  double* p;
  i64 gx, gz, sx;
  double& operator()(i64 i, i64 k) const { return p[(i + gx) + sx * (k + gz)]; }
};
inline F2 gview2(double* p, i64 nx, i64 nz, i64 gx, i64 gz) {
  F2 f;
  f.p = p; f.gx = gx; f.gz = gz; f.sx = nx + 1 + 2 * gx;
  (void)nz;
  return f;
}

inline double gather2(const F2& g, const Shape& a, const Shape& c, double acc) {
  for (int ll = c.lo; ll <= c.hi; ++ll)
    for (int jj = a.lo; jj <= a.hi; ++jj)
      acc = acc + a.s[jj - a.lo] * c.s[ll - c.lo] * g(a.i0 + jj, c.i0 + ll);
  return acc;
}

extern "C" {

// which: 0 = E, 1 = B.  Accumulates into f1, f2, f3.
void orc_geteb2dxz_energy_conserving_scalar(i64 which, i64 np, const double* xp,
                                            const double* zp, double* f1, double* f2,
                                            double* f3, double xmin, double zmin, double dx,
                                            double dz, i64 nx, i64 nz, i64 nxguard,
                                            i64 nzguard, i64 order, double* g1_, double* g2_,
                                            double* g3_, i64 l_lower_order_in_v, i64 l_nodal) {
  F2 g1 = gview2(g1_, nx, nz, nxguard, nzguard), g2 = gview2(g2_, nx, nz, nxguard, nzguard),
     g3 = gview2(g3_, nx, nz, nxguard, nzguard);
  const double ss = l_nodal ? 0.0 : 0.5;
  const bool lower = l_lower_order_in_v != 0;
  const double dxi = 1.0 / dx, dzi = 1.0 / dz;
  for (i64 ip = 0; ip < np; ++ip) {
    const double x = (xp[ip] - xmin) * dxi, z = (zp[ip] - zmin) * dzi;
    Shape nxs, nzs, sxs, szs;
    node_shape((int)order, x, nxs); node_shape((int)order, z, nzs);
    stag_shape((int)order, lower, ss, x, sxs); stag_shape((int)order, lower, ss, z, szs);
    if (which == 0) {
      f1[ip] = gather2(g1, sxs, nzs, f1[ip]);
      f2[ip] = gather2(g2, nxs, nzs, f2[ip]);
      f3[ip] = gather2(g3, nxs, szs, f3[ip]);
    } else {
      f1[ip] = gather2(g1, nxs, szs, f1[ip]);
      f2[ip] = gather2(g2, sxs, szs, f2[ip]);
      f3[ip] = gather2(g3, sxs, nzs, f3[ip]);
    }
  }
}

// pxr_depose_jxjyjz_esirkepov2d_{1_1,2_2,3_3} (esirkepov_2d.F90:452-623,
// :666-842, :843-1082), with l_particles_weight and no RZ or symmetry
// options: new shape sx0 at x, old shape sx at xold = x - dt/dx*vx shifted by
// the node difference; Jx prefix-summed along x inside each z row, Jz along z
// per x column, Jy deposited directly (the 2-D Esirkepov out-of-plane
// current).  The shape constants 1/6, 2/3 and the 1/3 of Jy are the
// reference's default-real (single precision) values.
void orc_depose_jxjyjz_esirkepov2d(i64 order, double* jx_, double* jy_, double* jz_, i64 np,
                                   const double* xp, const double* zp, const double* uxp,
                                   const double* uyp, const double* uzp, const double* gaminv,
                                   const double* w, double q, double xmin, double zmin,
                                   double dt, double dx, double dz, i64 nx, i64 nz,
                                   i64 nxguard, i64 nzguard) {
  F2 jx = gview2(jx_, nx, nz, nxguard, nzguard), jy = gview2(jy_, nx, nz, nxguard, nzguard),
     jz = gview2(jz_, nx, nz, nxguard, nzguard);
  const double onesixth_r = (double)(1.0f / 6.0f), twothird_r = (double)(2.0f / 3.0f);
  const double onethird_r = (double)(1.0f / 3.0f);
  const double dxi = 1.0 / dx, dzi = 1.0 / dz;
  const double dtsdx0 = dt * dxi, dtsdz0 = dt * dzi;
  const double invvol = 1.0 / (dx * dz), invdtdx = 1.0 / (dt * dz), invdtdz = 1.0 / (dt * dx);
  // (-2:3) arrays at offset +2
  double sx_[6], sz_[6], sx0_[6], sz0_[6], dsx_[6], dsz_[6], sdzk_[6], sdzkm1_[6];
  double *sx = sx_ + 2, *sz = sz_ + 2, *sx0 = sx0_ + 2, *sz0 = sz0_ + 2, *dsx = dsx_ + 2,
         *dsz = dsz_ + 2, *sdzk = sdzk_ + 2, *sdzkm1 = sdzkm1_ + 2;
  for (int t = 0; t < 6; ++t) { sx0_[t] = sz0_[t] = sdzk_[t] = sdzkm1_[t] = 0.0; }
  double sdxi = 0.0, sdxim1 = 0.0;
  auto shape = [&](double xint, double* s, int off) {
    if (order == 1) {
      s[0 + off] = 1.0 - xint; s[1 + off] = xint;
    } else if (order == 2) {
      const double xs = xint * xint;
      s[-1 + off] = 0.5 * (0.5 - xint) * (0.5 - xint);
      s[0 + off] = 0.75 - xs;
      s[1 + off] = 0.5 * (0.5 + xint) * (0.5 + xint);
    } else {
      const double ox = 1.0 - xint, xs = xint * xint, oxs = ox * ox;
      s[-1 + off] = onesixth_r * oxs * ox;
      s[0 + off] = twothird_r - xs * (1.0 - xint * 0.5);
      s[1 + off] = twothird_r - oxs * (1.0 - ox * 0.5);
      s[2 + off] = onesixth_r * xs * xint;
    }
  };
  auto node = [&](double v) -> i64 { return order == 2 ? fnint(v) : ffloor(v); };
  const int a = order == 1 ? 0 : 1, b = order == 3 ? 2 : 1;
  for (i64 ip = 0; ip < np; ++ip) {
    for (int t = 0; t < 6; ++t) { sx_[t] = sz_[t] = 0.0; }
    if (order != 2) for (int t = 0; t < 6; ++t) { sx0_[t] = sz0_[t] = 0.0; }
    const double x = (xp[ip] - xmin) * dxi, z = (zp[ip] - zmin) * dzi;
    const double vx = uxp[ip] * gaminv[ip], vy = uyp[ip] * gaminv[ip],
                 vz = uzp[ip] * gaminv[ip];
    const double xold = x - dtsdx0 * vx, zold = z - dtsdz0 * vz;
    const double wq = q * w[ip], wqx = wq * invdtdx, wqz = wq * invdtdz;
    const i64 iixp0 = node(x), ikxp0 = node(z);
    shape(x - iixp0, sx0, 0);
    shape(z - ikxp0, sz0, 0);
    const i64 iixp = node(xold), ikxp = node(zold);
    const int dix = (int)(iixp - iixp0), diz = (int)(ikxp - ikxp0);
    shape(xold - iixp, sx, dix);
    shape(zold - ikxp, sz, diz);
    for (int t = 0; t < 6; ++t) { dsx_[t] = sx_[t] - sx0_[t]; dsz_[t] = sz_[t] - sz0_[t]; }
    const int ixmin = std::min(0, dix) - a, ixmax = std::max(0, dix) + b;
    const int izmin = std::min(0, diz) - a, izmax = std::max(0, diz) + b;
    for (int k = izmin; k <= izmax; ++k) {
      for (int i = ixmin; i <= ixmax; ++i) {
        const i64 ic = iixp0 + i, kc = ikxp0 + k;
        if (i < ixmax) {
          sdxi = wqx * dsx[i] * (sz0[k] + 0.5 * dsz[k]);
          if (i > ixmin) sdxi = sdxi + sdxim1;
          jx(ic, kc) = jx(ic, kc) + sdxi;
        }
        jy(ic, kc) = jy(ic, kc) + wq * vy * invvol *
                                      ((sz0[k] + 0.5 * dsz[k]) * sx0[i] +
                                       (0.5 * sz0[k] + onethird_r * dsz[k]) * dsx[i]);
        if (k < izmax) {
          sdzk[i] = wqz * dsz[k] * (sx0[i] + 0.5 * dsx[i]);
          if (k > izmin) sdzk[i] = sdzk[i] + sdzkm1[i];
          jz(ic, kc) = jz(ic, kc) + sdzk[i];
        }
        sdxim1 = sdxi;
      }
      for (int t = 0; t < 6; ++t) sdzkm1_[t] = sdzk_[t];
    }
  }
}

// pxrpush_em2d_evec / pxrpush_em2d_bvec (yee.F90:216-310, :912-994): the
// order-2 Yee update in x-z; bnds: [xlo(2) xhi(2) ylo(2) yhi(2) zlo(2)
// zhi(2)] loop ranges of the three components; every array (-g:n+g)^2.
void orc_pxrpush_em2d_evec(const i64* bnds, double* ex_, double* ey_, double* ez_, double* bx_,
                           double* by_, double* bz_, double* jx_, double* jy_, double* jz_,
                           i64 nx, i64 nz, i64 g, double mudt, double dtsdx, double dtsdz) {
  F2 Ex = gview2(ex_, nx, nz, g, g), Ey = gview2(ey_, nx, nz, g, g), Ez = gview2(ez_, nx, nz, g, g),
     Bx = gview2(bx_, nx, nz, g, g), By = gview2(by_, nx, nz, g, g), Bz = gview2(bz_, nx, nz, g, g),
     Jx = gview2(jx_, nx, nz, g, g), Jy = gview2(jy_, nx, nz, g, g), Jz = gview2(jz_, nx, nz, g, g);
  const i64 *xlo = bnds, *xhi = bnds + 2, *ylo = bnds + 4, *yhi = bnds + 6, *zlo = bnds + 8,
            *zhi = bnds + 10;
  for (i64 k = xlo[1]; k <= xhi[1]; ++k)
    for (i64 j = xlo[0]; j <= xhi[0]; ++j)
      Ex(j, k) = Ex(j, k) - dtsdz * (By(j, k) - By(j, k - 1)) - mudt * Jx(j, k);
  for (i64 k = ylo[1]; k <= yhi[1]; ++k)
    for (i64 j = ylo[0]; j <= yhi[0]; ++j)
      Ey(j, k) = Ey(j, k) - dtsdx * (Bz(j, k) - Bz(j - 1, k)) + dtsdz * (Bx(j, k) - Bx(j, k - 1)) -
                 mudt * Jy(j, k);
  for (i64 k = zlo[1]; k <= zhi[1]; ++k)
    for (i64 j = zlo[0]; j <= zhi[0]; ++j)
      Ez(j, k) = Ez(j, k) + dtsdx * (By(j, k) - By(j - 1, k)) - mudt * Jz(j, k);
}

void orc_pxrpush_em2d_bvec(const i64* bnds, double* ex_, double* ey_, double* ez_, double* bx_,
                           double* by_, double* bz_, i64 nx, i64 nz, i64 g, double dtsdx,
                           double dtsdz) {
  F2 Ex = gview2(ex_, nx, nz, g, g), Ey = gview2(ey_, nx, nz, g, g), Ez = gview2(ez_, nx, nz, g, g),
     Bx = gview2(bx_, nx, nz, g, g), By = gview2(by_, nx, nz, g, g), Bz = gview2(bz_, nx, nz, g, g);
  const i64 *xlo = bnds, *xhi = bnds + 2, *ylo = bnds + 4, *yhi = bnds + 6, *zlo = bnds + 8,
            *zhi = bnds + 10;
  for (i64 k = xlo[1]; k <= xhi[1]; ++k)
    for (i64 j = xlo[0]; j <= xhi[0]; ++j)
      Bx(j, k) = Bx(j, k) + dtsdz * (Ey(j, k + 1) - Ey(j, k));
  for (i64 k = ylo[1]; k <= yhi[1]; ++k)
    for (i64 j = ylo[0]; j <= yhi[0]; ++j)
      By(j, k) = By(j, k) + dtsdx * (Ez(j + 1, k) - Ez(j, k)) - dtsdz * (Ex(j, k + 1) - Ex(j, k));
  for (i64 k = zlo[1]; k <= zhi[1]; ++k)
    for (i64 j = zlo[0]; j <= zhi[0]; ++j)
      Bz(j, k) = Bz(j, k) - dtsdx * (Ey(j + 1, k) - Ey(j, k));
}

// pxr_pushxz (boris_2d.F90:42-60)
void orc_pushxz(i64 np, double* xp, double* zp, const double* uxp, const double* uzp,
                const double* gaminv, double dt) {
  for (i64 ip = 0; ip < np; ++ip) {
    xp[ip] = xp[ip] + uxp[ip] * gaminv[ip] * dt;
    zp[ip] = zp[ip] + uzp[ip] * gaminv[ip] * dt;
  }
}

}  // extern "C"

// ----------------------------------------------------------------------------
// Esirkepov current deposition (accumulates into jx, jy, jz).
// src/particle_deposition/current_deposition/esirkepov/esirkepov_3d.F90:
//   depose_jxjyjz_esirkepov_1_1_1  :82-239
//   depose_jxjyjz_esirkepov_2_2_2  :1734-1918
//   depose_jxjyjz_esirkepov_3_3_3  :3263-3464
//   pxr_depose_jxjyjz_esirkepov_n  :3480-3848
// Grids are (-ng : nvalid+ng-1) = (-ng : n+ng) per axis.  sx0 holds the shape
// at the new position x, sx the shape at xold = x - dt/dx*ux*gaminv, shifted
// by the cell difference; currents are prefix sums along i (Jx), j (Jy),
// k (Jz) inside the (min(0,d)-a : max(0,d)+b) box.
// ----------------------------------------------------------------------------
void orc_depose_jxjyjz_esirkepov_1_1_1(
    double* jx_, double* jy_, double* jz_, i64 np, const double* xp,
    const double* yp, const double* zp, const double* uxp, const double* uyp,
    const double* uzp, const double* gaminv, const double* w, double q,
    double xmin, double ymin, double zmin, double dt, double dx, double dy,
    double dz, i64 nx, i64 ny, i64 nz, i64 nxguard, i64 nyguard, i64 nzguard) {
  F3 jx = gview(jx_, nx, ny, nz, nxguard, nyguard, nzguard);
  F3 jy = gview(jy_, nx, ny, nz, nxguard, nyguard, nzguard);
  F3 jz = gview(jz_, nx, ny, nz, nxguard, nyguard, nzguard);
  const double dxi = 1.0 / dx, dyi = 1.0 / dy, dzi = 1.0 / dz;
  const double dtsdx0 = dt * dxi, dtsdy0 = dt * dyi, dtsdz0 = dt * dzi;
  const double invdtdx = 1.0 / (dt * dy * dz);
  const double invdtdy = 1.0 / (dt * dx * dz);
  const double invdtdz = 1.0 / (dt * dx * dy);
  const double onethird = 1.0 / 3.0;
  // (-1:2) arrays at offset +1
  double sx_[4], sy_[4], sz_[4], sx0_[4], sy0_[4], sz0_[4];
  double *sx = sx_ + 1, *sy = sy_ + 1, *sz = sz_ + 1;
  double *sx0 = sx0_ + 1, *sy0 = sy0_ + 1, *sz0 = sz0_ + 1;
  double sdxi = 0.0, sdxim1 = 0.0;
  double sdyj_[4] = {0, 0, 0, 0}, sdyjm1_[4] = {0, 0, 0, 0};
  double sdzk_[4][4] = {}, sdzkm1_[4][4] = {};
  double *sdyj = sdyj_ + 1, *sdyjm1 = sdyjm1_ + 1;
  for (i64 ip = 0; ip < np; ++ip) {
    for (int t = 0; t < 4; ++t) sx_[t] = sy_[t] = sz_[t] = sx0_[t] = sy0_[t] = sz0_[t] = 0.0;
    double x = (xp[ip] - xmin) * dxi, y = (yp[ip] - ymin) * dyi, z = (zp[ip] - zmin) * dzi;
    double xold = x - dtsdx0 * uxp[ip] * gaminv[ip];
    double yold = y - dtsdy0 * uyp[ip] * gaminv[ip];
    double zold = z - dtsdz0 * uzp[ip] * gaminv[ip];
    double wq = q * w[ip];
    i64 iixp0 = ffloor(x), ijxp0 = ffloor(y), ikxp0 = ffloor(z);
    sx0[0] = 1.0 - (x - iixp0); sx0[1] = x - iixp0;
    sy0[0] = 1.0 - (y - ijxp0); sy0[1] = y - ijxp0;
    sz0[0] = 1.0 - (z - ikxp0); sz0[1] = z - ikxp0;
    i64 iixp = ffloor(xold), ijxp = ffloor(yold), ikxp = ffloor(zold);
    sx[0 + iixp - iixp0] = 1.0 - (xold - iixp); sx[1 + iixp - iixp0] = xold - iixp;
    sy[0 + ijxp - ijxp0] = 1.0 - (yold - ijxp); sy[1 + ijxp - ijxp0] = yold - ijxp;
    sz[0 + ikxp - ikxp0] = 1.0 - (zold - ikxp); sz[1 + ikxp - ikxp0] = zold - ikxp;
    i64 ixmin = std::min<i64>(0, iixp - iixp0), ixmax = std::max<i64>(0, iixp - iixp0) + 1;
    i64 iymin = std::min<i64>(0, ijxp - ijxp0), iymax = std::max<i64>(0, ijxp - ijxp0) + 1;
    i64 izmin = std::min<i64>(0, ikxp - ikxp0), izmax = std::max<i64>(0, ikxp - ikxp0) + 1;
    for (i64 k = izmin; k <= izmax; ++k) {
      for (i64 j = iymin; j <= iymax; ++j) {
        for (i64 i = ixmin; i <= ixmax; ++i) {
          i64 ic = iixp0 + i, jc = ijxp0 + j, kc = ikxp0 + k;
          if (i < ixmax) {
            sdxi = wq * invdtdx * (sx[i] - sx0[i]) *
                   ((sy0[j] + 0.5 * (sy[j] - sy0[j])) * sz0[k] +
                    (0.5 * sy0[j] + onethird * (sy[j] - sy0[j])) * (sz[k] - sz0[k]));
            if (i > ixmin) sdxi = sdxi + sdxim1;
            jx(ic, jc, kc) = jx(ic, jc, kc) + sdxi;
          }
          if (j < iymax) {
            sdyj[i] = wq * invdtdy * (sy[j] - sy0[j]) *
                      ((sz0[k] + 0.5 * (sz[k] - sz0[k])) * sx0[i] +
                       (0.5 * sz0[k] + onethird * (sz[k] - sz0[k])) * (sx[i] - sx0[i]));
            if (j > iymin) sdyj[i] = sdyj[i] + sdyjm1[i];
            jy(ic, jc, kc) = jy(ic, jc, kc) + sdyj[i];
          }
          if (k < izmax) {
            sdzk_[i + 1][j + 1] = wq * invdtdz * (sz[k] - sz0[k]) *
                                  ((sx0[i] + 0.5 * (sx[i] - sx0[i])) * sy0[j] +
                                   (0.5 * sx0[i] + onethird * (sx[i] - sx0[i])) * (sy[j] - sy0[j]));
            if (k > izmin) sdzk_[i + 1][j + 1] = sdzk_[i + 1][j + 1] + sdzkm1_[i + 1][j + 1];
            jz(ic, jc, kc) = jz(ic, jc, kc) + sdzk_[i + 1][j + 1];
          }
          sdxim1 = sdxi;
        }
        std::memcpy(sdyjm1_, sdyj_, sizeof(sdyj_));
      }
      std::memcpy(sdzkm1_, sdzk_, sizeof(sdzk_));
    }
  }
}

// Orders 2 and 3 share the same loop body; only the shape functions, the
// node rounding (nint for order 2, floor for order 3) and the box bounds
// differ.  Arrays (-2:3) at offset +2.
static void esirkepov_23(int order, double* jx_, double* jy_, double* jz_, i64 np,
                         const double* xp, const double* yp, const double* zp,
                         const double* uxp, const double* uyp, const double* uzp,
                         const double* gaminv, const double* w, double q,
                         double xmin, double ymin, double zmin, double dt,
                         double dx, double dy, double dz, i64 nx, i64 ny, i64 nz,
                         i64 nxguard, i64 nyguard, i64 nzguard) {
  F3 jx = gview(jx_, nx, ny, nz, nxguard, nyguard, nzguard);
  F3 jy = gview(jy_, nx, ny, nz, nxguard, nyguard, nzguard);
  F3 jz = gview(jz_, nx, ny, nz, nxguard, nyguard, nzguard);
  const double dxi = 1.0 / dx, dyi = 1.0 / dy, dzi = 1.0 / dz;
  const double dtsdx0 = dt * dxi, dtsdy0 = dt * dyi, dtsdz0 = dt * dzi;
  const double invdtdx = 1.0 / (dt * dy * dz);
  const double invdtdy = 1.0 / (dt * dx * dz);
  const double invdtdz = 1.0 / (dt * dx * dy);
  const int O = 2;  // offset for (-2:3)
  double sx[6], sy[6], sz[6], sx0[6], sy0[6], sz0[6], dsx[6], dsy[6], dsz[6];
  double sdxi = 0.0, sdxim1 = 0.0;
  double sdyj[6] = {}, sdyjm1[6] = {};
  double sdzk[6][6] = {}, sdzkm1[6][6] = {};
  auto quad = [](double* s, int base, double xi) {
    double xs = xi * xi;
    s[base - 1] = 0.5 * sq(0.5 - xi);
    s[base] = 0.75 - xs;
    s[base + 1] = 0.5 * sq(0.5 + xi);
  };
  auto cubic = [](double* s, int base, double xi) {
    double ox = 1.0 - xi, xs = xi * xi, oxs = ox * ox;
    s[base - 1] = onesixth * oxs * ox;
    s[base] = twothird - xs * (1.0 - xi / 2.0);
    s[base + 1] = twothird - oxs * (1.0 - ox / 2.0);
    s[base + 2] = onesixth * xs * xi;
  };
  auto rnd = [order](double v) -> i64 { return order == 2 ? fnint(v) : ffloor(v); };
  const i64 up = (order == 2) ? 1 : 2;
  for (i64 ip = 0; ip < np; ++ip) {
    for (int t = 0; t < 6; ++t) sx[t] = sy[t] = sz[t] = sx0[t] = sy0[t] = sz0[t] = 0.0;
    double x = (xp[ip] - xmin) * dxi, y = (yp[ip] - ymin) * dyi, z = (zp[ip] - zmin) * dzi;
    double vx = uxp[ip] * gaminv[ip], vy = uyp[ip] * gaminv[ip], vz = uzp[ip] * gaminv[ip];
    double xold = x - dtsdx0 * vx, yold = y - dtsdy0 * vy, zold = z - dtsdz0 * vz;
    double wq = q * w[ip];
    double wqx = wq * invdtdx, wqy = wq * invdtdy, wqz = wq * invdtdz;
    i64 iixp0 = rnd(x), ijxp0 = rnd(y), ikxp0 = rnd(z);
    if (order == 2) {
      quad(sx0, O, x - iixp0); quad(sy0, O, y - ijxp0); quad(sz0, O, z - ikxp0);
    } else {
      cubic(sx0, O, x - iixp0); cubic(sy0, O, y - ijxp0); cubic(sz0, O, z - ikxp0);
    }
    i64 iixp = rnd(xold), ijxp = rnd(yold), ikxp = rnd(zold);
    i64 dix = iixp - iixp0, diy = ijxp - ijxp0, diz = ikxp - ikxp0;
    if (order == 2) {
      quad(sx, O + (int)dix, xold - iixp); quad(sy, O + (int)diy, yold - ijxp);
      quad(sz, O + (int)diz, zold - ikxp);
    } else {
      cubic(sx, O + (int)dix, xold - iixp); cubic(sy, O + (int)diy, yold - ijxp);
      cubic(sz, O + (int)diz, zold - ikxp);
    }
    for (int t = 0; t < 6; ++t) {
      dsx[t] = sx[t] - sx0[t]; dsy[t] = sy[t] - sy0[t]; dsz[t] = sz[t] - sz0[t];
    }
    i64 ixmin = std::min<i64>(0, dix) - 1, ixmax = std::max<i64>(0, dix) + up;
    i64 iymin = std::min<i64>(0, diy) - 1, iymax = std::max<i64>(0, diy) + up;
    i64 izmin = std::min<i64>(0, diz) - 1, izmax = std::max<i64>(0, diz) + up;
    for (i64 k = izmin; k <= izmax; ++k) {
      for (i64 j = iymin; j <= iymax; ++j) {
        for (i64 i = ixmin; i <= ixmax; ++i) {
          i64 ic = iixp0 + i, jc = ijxp0 + j, kc = ikxp0 + k;
          int I = (int)i + O, J = (int)j + O, K = (int)k + O;
          if (i < ixmax) {
            sdxi = wqx * dsx[I] * ((sy0[J] + 0.5 * dsy[J]) * sz0[K] +
                                   (0.5 * sy0[J] + 1.0 / 3.0 * dsy[J]) * dsz[K]);
            if (i > ixmin) sdxi = sdxi + sdxim1;
            jx(ic, jc, kc) = jx(ic, jc, kc) + sdxi;
          }
          if (j < iymax) {
            sdyj[I] = wqy * dsy[J] * ((sz0[K] + 0.5 * dsz[K]) * sx0[I] +
                                      (0.5 * sz0[K] + 1.0 / 3.0 * dsz[K]) * dsx[I]);
            if (j > iymin) sdyj[I] = sdyj[I] + sdyjm1[I];
            jy(ic, jc, kc) = jy(ic, jc, kc) + sdyj[I];
          }
          if (k < izmax) {
            sdzk[I][J] = wqz * dsz[K] * ((sx0[I] + 0.5 * dsx[I]) * sy0[J] +
                                         (0.5 * sx0[I] + 1.0 / 3.0 * dsx[I]) * dsy[J]);
            if (k > izmin) sdzk[I][J] = sdzk[I][J] + sdzkm1[I][J];
            jz(ic, jc, kc) = jz(ic, jc, kc) + sdzk[I][J];
          }
          sdxim1 = sdxi;
        }
        std::memcpy(sdyjm1, sdyj, sizeof(sdyj));
      }
      std::memcpy(sdzkm1, sdzk, sizeof(sdzk));
    }
  }
}

void orc_depose_jxjyjz_esirkepov_2_2_2(
    double* jx, double* jy, double* jz, i64 np, const double* xp, const double* yp,
    const double* zp, const double* uxp, const double* uyp, const double* uzp,
    const double* gaminv, const double* w, double q, double xmin, double ymin,
    double zmin, double dt, double dx, double dy, double dz, i64 nx, i64 ny,
    i64 nz, i64 nxguard, i64 nyguard, i64 nzguard) {
  esirkepov_23(2, jx, jy, jz, np, xp, yp, zp, uxp, uyp, uzp, gaminv, w, q, xmin,
               ymin, zmin, dt, dx, dy, dz, nx, ny, nz, nxguard, nyguard, nzguard);
}

void orc_depose_jxjyjz_esirkepov_3_3_3(
    double* jx, double* jy, double* jz, i64 np, const double* xp, const double* yp,
    const double* zp, const double* uxp, const double* uyp, const double* uzp,
    const double* gaminv, const double* w, double q, double xmin, double ymin,
    double zmin, double dt, double dx, double dy, double dz, i64 nx, i64 ny,
    i64 nz, i64 nxguard, i64 nyguard, i64 nzguard) {
  esirkepov_23(3, jx, jy, jz, np, xp, yp, zp, uxp, uyp, uzp, gaminv, w, q, xmin,
               ymin, zmin, dt, dx, dy, dz, nx, ny, nz, nxguard, nyguard, nzguard);
}

// Arbitrary-order generic form (orders 0..3 per axis), with the position
// reconstructed as xold + dt/dx*v and one sub-cycle (ncells = 1), as in
// esirkepov_3d.F90:3480-3848.  l_particles_weight = .TRUE., l4symtry = .FALSE.
// (the values depose_jxjyjz_esirkepov passes, current_deposition_manager_3d.F90:75-104).
void orc_pxr_depose_jxjyjz_esirkepov_n(
    double* jx_, double* jy_, double* jz_, i64 np, const double* xp,
    const double* yp, const double* zp, const double* uxp, const double* uyp,
    const double* uzp, const double* gaminv, const double* w, double q,
    double xmin, double ymin, double zmin, double dt, double dx, double dy,
    double dz, i64 nx, i64 ny, i64 nz, i64 nxguard, i64 nyguard, i64 nzguard,
    i64 nox, i64 noy, i64 noz, double clight) {
  F3 jx = gview(jx_, nx, ny, nz, nxguard, nyguard, nzguard);
  F3 jy = gview(jy_, nx, ny, nz, nxguard, nyguard, nzguard);
  F3 jz = gview(jz_, nx, ny, nz, nxguard, nyguard, nzguard);
  const i64 ndtodx = (i64)(clight * dt / dx), ndtody = (i64)(clight * dt / dy),
            ndtodz = (i64)(clight * dt / dz);
  const double dxi = 1.0 / dx, dyi = 1.0 / dy, dzi = 1.0 / dz;
  const double dtsdx0 = dt * dxi, dtsdy0 = dt * dyi, dtsdz0 = dt * dzi;
  const double invdtdx = 1.0 / (dt * dy * dz);
  const double invdtdy = 1.0 / (dt * dx * dz);
  const double invdtdz = 1.0 / (dt * dx * dy);
  const i64 xl = -(nox / 2) - 1 - ndtodx, xu = (nox + 1) / 2 + 1 + ndtodx;
  const i64 yl = -(noy / 2) - 1 - ndtody, yu = (noy + 1) / 2 + 1 + ndtody;
  const i64 zl = -(noz / 2) - 1 - ndtodz, zu = (noz + 1) / 2 + 1 + ndtodz;
  const i64 NX = xu - xl + 1, NY = yu - yl + 1, NZ = zu - zl + 1;
  std::vector<double> sdx(NX * NY * NZ, 0.0), sdy(NX * NY * NZ, 0.0), sdz(NX * NY * NZ, 0.0);
  std::vector<double> sxv(NX), sx0v(NX, 0.0), dsxv(NX), syv(NY), sy0v(NY, 0.0), dsyv(NY),
      szv(NZ), sz0v(NZ, 0.0), dszv(NZ);
  double *sx = sxv.data() - xl, *sx0 = sx0v.data() - xl, *dsx = dsxv.data() - xl;
  double *sy = syv.data() - yl, *sy0 = sy0v.data() - yl, *dsy = dsyv.data() - yl;
  double *sz = szv.data() - zl, *sz0 = sz0v.data() - zl, *dsz = dszv.data() - zl;
  auto S = [&](std::vector<double>& a, i64 i, i64 j, i64 k) -> double& {
    return a[(i - xl) + NX * ((j - yl) + NY * (k - zl))];
  };
  auto shape = [](i64 no, double* s, i64 base, double xi) {
    switch (no) {
      case 0: s[base] = 1.0; break;
      case 1: s[base] = 1.0 - xi; s[base + 1] = xi; break;
      case 2: {
        double xs = xi * xi;
        s[base - 1] = 0.5 * sq(0.5 - xi); s[base] = 0.75 - xs; s[base + 1] = 0.5 * sq(0.5 + xi);
        break;
      }
      case 3: {
        double ox = 1.0 - xi, xs = xi * xi, oxs = ox * ox;
        s[base - 1] = onesixth * oxs * ox;
        s[base] = twothird - xs * (1.0 - xi / 2.0);
        s[base + 1] = twothird - oxs * (1.0 - ox / 2.0);
        s[base + 2] = onesixth * xs * xi;
        break;
      }
    }
  };
  auto rnd = [](i64 no, double v) -> i64 { return (no == 2 * (no / 2)) ? fnint(v) : ffloor(v); };
  for (i64 ip = 0; ip < np; ++ip) {
    double x = (xp[ip] - xmin) * dxi, y = (yp[ip] - ymin) * dyi, z = (zp[ip] - zmin) * dzi;
    double vx = uxp[ip] * gaminv[ip], vy = uyp[ip] * gaminv[ip], vz = uzp[ip] * gaminv[ip];
    double xold = x - dtsdx0 * vx, yold = y - dtsdy0 * vy, zold = z - dtsdz0 * vz;
    const i64 ncells = 1;
    double dtsdx = dtsdx0 / ncells, dtsdy = dtsdy0 / ncells, dtsdz = dtsdz0 / ncells;
    x = xold; y = yold; z = zold;
    for (i64 icell = 1; icell <= ncells; ++icell) {
      xold = x; yold = y; zold = z;
      x = x + dtsdx * vx; y = y + dtsdy * vy; z = z + dtsdz * vz;
      double wq = q * w[ip];
      double wqx = wq * invdtdx, wqy = wq * invdtdy, wqz = wq * invdtdz;
      i64 iixp0 = rnd(nox, x), ijxp0 = rnd(noy, y), ikxp0 = rnd(noz, z);
      shape(nox, sx0, 0, x - iixp0); shape(noy, sy0, 0, y - ijxp0); shape(noz, sz0, 0, z - ikxp0);
      i64 iixp = rnd(nox, xold), ijxp = rnd(noy, yold), ikxp = rnd(noz, zold);
      i64 dix = iixp - iixp0, diy = ijxp - ijxp0, diz = ikxp - ikxp0;
      std::fill(sxv.begin(), sxv.end(), 0.0);
      std::fill(syv.begin(), syv.end(), 0.0);
      std::fill(szv.begin(), szv.end(), 0.0);
      shape(nox, sx, dix, xold - iixp); shape(noy, sy, diy, yold - ijxp); shape(noz, sz, diz, zold - ikxp);
      for (i64 t = xl; t <= xu; ++t) dsx[t] = sx[t] - sx0[t];
      for (i64 t = yl; t <= yu; ++t) dsy[t] = sy[t] - sy0[t];
      for (i64 t = zl; t <= zu; ++t) dsz[t] = sz[t] - sz0[t];
      i64 ixmin = std::min<i64>(0, dix) - nox / 2, ixmax = std::max<i64>(0, dix) + (nox + 1) / 2;
      i64 iymin = std::min<i64>(0, diy) - noy / 2, iymax = std::max<i64>(0, diy) + (noy + 1) / 2;
      i64 izmin = std::min<i64>(0, diz) - noz / 2, izmax = std::max<i64>(0, diz) + (noz + 1) / 2;
      for (i64 k = izmin; k <= izmax; ++k)
        for (i64 j = iymin; j <= iymax; ++j)
          for (i64 i = ixmin; i <= ixmax; ++i) {
            i64 ic = iixp0 + i, jc = ijxp0 + j, kc = ikxp0 + k;
            if (i < ixmax) {
              S(sdx, i, j, k) = wqx * dsx[i] * ((sy0[j] + 0.5 * dsy[j]) * sz0[k] +
                                                (0.5 * sy0[j] + 1.0 / 3.0 * dsy[j]) * dsz[k]);
              if (i > ixmin) S(sdx, i, j, k) = S(sdx, i, j, k) + S(sdx, i - 1, j, k);
              jx(ic, jc, kc) = jx(ic, jc, kc) + S(sdx, i, j, k);
            }
            if (j < iymax) {
              S(sdy, i, j, k) = wqy * dsy[j] * ((sz0[k] + 0.5 * dsz[k]) * sx0[i] +
                                                (0.5 * sz0[k] + 1.0 / 3.0 * dsz[k]) * dsx[i]);
              if (j > iymin) S(sdy, i, j, k) = S(sdy, i, j, k) + S(sdy, i, j - 1, k);
              jy(ic, jc, kc) = jy(ic, jc, kc) + S(sdy, i, j, k);
            }
            if (k < izmax) {
              S(sdz, i, j, k) = wqz * dsz[k] * ((sx0[i] + 0.5 * dsx[i]) * sy0[j] +
                                                (0.5 * sx0[i] + 1.0 / 3.0 * dsx[i]) * dsy[j]);
              if (k > izmin) S(sdz, i, j, k) = S(sdz, i, j, k) + S(sdz, i, j, k - 1);
              jz(ic, jc, kc) = jz(ic, jc, kc) + S(sdz, i, j, k);
            }
          }
    }
  }
}

// Dispatch of depose_jxjyjz_generic for current_depo_algo = 0 / 1
// (current_deposition_manager_3d.F90:106-208).
void orc_depose_jxjyjz(double* jx, double* jy, double* jz, i64 np, const double* xp,
                       const double* yp, const double* zp, const double* uxp,
                       const double* uyp, const double* uzp, const double* gaminv,
                       const double* w, double q, double xmin, double ymin,
                       double zmin, double dt, double dx, double dy, double dz,
                       i64 nx, i64 ny, i64 nz, i64 nxguard, i64 nyguard,
                       i64 nzguard, i64 nox, i64 noy, i64 noz,
                       i64 current_depo_algo, double clight) {
  if (current_depo_algo == 0 && nox == noy && noy == noz && nox >= 1 && nox <= 3) {
    if (nox == 1)
      orc_depose_jxjyjz_esirkepov_1_1_1(jx, jy, jz, np, xp, yp, zp, uxp, uyp, uzp, gaminv,
                                        w, q, xmin, ymin, zmin, dt, dx, dy, dz, nx, ny,
                                        nz, nxguard, nyguard, nzguard);
    else
      esirkepov_23((int)nox, jx, jy, jz, np, xp, yp, zp, uxp, uyp, uzp, gaminv, w, q,
                   xmin, ymin, zmin, dt, dx, dy, dz, nx, ny, nz, nxguard, nyguard,
                   nzguard);
  } else {
    orc_pxr_depose_jxjyjz_esirkepov_n(jx, jy, jz, np, xp, yp, zp, uxp, uyp, uzp, gaminv,
                                      w, q, xmin, ymin, zmin, dt, dx, dy, dz, nx, ny, nz,
                                      nxguard, nyguard, nzguard, nox, noy, noz, clight);
  }
}

// ----------------------------------------------------------------------------
// Charge deposition (node-centred rho, accumulates).
// src/particle_deposition/charge_deposition/charge_deposition_3d.F90:77-172
// (order 1), :174-322 (order 2), :324-... (order 3).
// ----------------------------------------------------------------------------
void orc_depose_rho_scalar(i64 order, double* rho_, i64 np, const double* xp,
                           const double* yp, const double* zp, const double* w,
                           double q, double xmin, double ymin, double zmin,
                           double dx, double dy, double dz, i64 nx, i64 ny, i64 nz,
                           i64 nxguard, i64 nyguard, i64 nzguard) {
  F3 rho = gview(rho_, nx, ny, nz, nxguard, nyguard, nzguard);
  const double dxi = 1.0 / dx, dyi = 1.0 / dy, dzi = 1.0 / dz;
  const double invvol = dxi * dyi * dzi;
  for (i64 ip = 0; ip < np; ++ip) {
    double x = (xp[ip] - xmin) * dxi, y = (yp[ip] - ymin) * dyi, z = (zp[ip] - zmin) * dzi;
    double wq = q * w[ip] * invvol;
    if (order == 1) {
      i64 j = ffloor(x), k = ffloor(y), l = ffloor(z);
      double xint = x - j, yint = y - k, zint = z - l;
      double sx[2] = {1.0 - xint, xint}, sy[2] = {1.0 - yint, yint}, sz[2] = {1.0 - zint, zint};
      // statement order of the Fortran: (j,k,l) (j+1,k,l) (j,k+1,l) (j+1,k+1,l) then l+1
      for (int c = 0; c <= 1; ++c)
        for (int b = 0; b <= 1; ++b)
          for (int a = 0; a <= 1; ++a)
            rho(j + a, k + b, l + c) = rho(j + a, k + b, l + c) + sx[a] * sy[b] * sz[c] * wq;
    } else if (order == 2) {
      i64 j = fnint(x), k = fnint(y), l = fnint(z);
      double xint = x - j, yint = y - k, zint = z - l;
      double xs = xint * xint, ys = yint * yint, zs = zint * zint;
      double sx[3] = {0.5 * sq(0.5 - xint), 0.75 - xs, 0.5 * sq(0.5 + xint)};
      double sy[3] = {0.5 * sq(0.5 - yint), 0.75 - ys, 0.5 * sq(0.5 + yint)};
      double sz[3] = {0.5 * sq(0.5 - zint) * wq, (0.75 - zs) * wq, 0.5 * sq(0.5 + zint) * wq};
      double sxy[9];
      for (int b = 0; b < 3; ++b)
        for (int a = 0; a < 3; ++a) sxy[a + 3 * b] = sx[a] * sy[b];
      for (int c = 0; c < 3; ++c)
        for (int b = 0; b < 3; ++b)
          for (int a = 0; a < 3; ++a)
            rho(j + a - 1, k + b - 1, l + c - 1) =
                rho(j + a - 1, k + b - 1, l + c - 1) + sxy[a + 3 * b] * sz[c];
    } else {
      i64 j = ffloor(x), k = ffloor(y), l = ffloor(z);
      double xint = x - j, yint = y - k, zint = z - l;
      double s[3][4];
      double v[3] = {xint, yint, zint};
      for (int d = 0; d < 3; ++d) {
        double xi = v[d], ox = 1.0 - xi, xs = xi * xi, oxs = ox * ox;
        s[d][0] = onesixth * oxs * ox;
        s[d][1] = twothird - xs * (1.0 - xi / 2.0);
        s[d][2] = twothird - oxs * (1.0 - ox / 2.0);
        s[d][3] = onesixth * xs * xi;
      }
      for (int c = 0; c < 4; ++c)
        for (int b = 0; b < 4; ++b)
          for (int a = 0; a < 4; ++a)
            rho(j + a - 1, k + b - 1, l + c - 1) =
                rho(j + a - 1, k + b - 1, l + c - 1) + s[0][a] * s[1][b] * s[2][c] * wq;
    }
  }
}

// ----------------------------------------------------------------------------
// Yee FDTD (order 2).  src/field_solvers/Maxwell/yee_solver/yee.F90:637-740
// (pxrpush_em3d_evec) and :1258-1347 (pxrpush_em3d_bvec).  Each array has its
// own (lo:hi) bounds; each component its own loop range.
// bnds: [xlo(3) xhi(3) ylo(3) yhi(3) zlo(3) zhi(3)]; alo/ahi: 9 (E) or 6 (B)
// arrays' bounds, 3 each, in argument order ex,ey,ez,bx,by,bz,jx,jy,jz.
// ----------------------------------------------------------------------------
// ----------------------------------------------------------------------------
// Arbitrary-order Yee pushes, yee.F90:46-123 (E) and :752-821 (B): for each
// node of [-nxs, nx+nxs] x ..., the sum over i = 1..min(norder/2, distance to
// the array's upper and lower ends) of dtsd(i) times the difference of the
// source field at +-i (staggered: ist = 1, the forward point shifted back by
// one for E, the backward one forward by one for B; nodal grid: ist = 0).
// All nine arrays (-guard:n+guard) per axis; dtsdx(norderx/2) etc.
// ----------------------------------------------------------------------------
static inline i64 nord_hi(i64 half, i64 n, i64 g, i64 j) {
  return std::min(std::min(half, (n - j) + g), j + g);
}

void orc_pxrpush_em3d_evec_norder(double* ex_, double* ey_, double* ez_, double* bx_,
                                  double* by_, double* bz_, double* jx_, double* jy_,
                                  double* jz_, double mudt, const double* dtsdx,
                                  const double* dtsdy, const double* dtsdz, i64 nx, i64 ny,
                                  i64 nz, i64 norderx, i64 nordery, i64 norderz, i64 nxguard,
                                  i64 nyguard, i64 nzguard, i64 nxs, i64 nys, i64 nzs,
                                  i64 l_nodalgrid) {
  F3 Ex = gview(ex_, nx, ny, nz, nxguard, nyguard, nzguard);
  F3 Ey = gview(ey_, nx, ny, nz, nxguard, nyguard, nzguard);
  F3 Ez = gview(ez_, nx, ny, nz, nxguard, nyguard, nzguard);
  F3 Bx = gview(bx_, nx, ny, nz, nxguard, nyguard, nzguard);
  F3 By = gview(by_, nx, ny, nz, nxguard, nyguard, nzguard);
  F3 Bz = gview(bz_, nx, ny, nz, nxguard, nyguard, nzguard);
  F3 Jx = gview(jx_, nx, ny, nz, nxguard, nyguard, nzguard);
  F3 Jy = gview(jy_, nx, ny, nz, nxguard, nyguard, nzguard);
  F3 Jz = gview(jz_, nx, ny, nz, nxguard, nyguard, nzguard);
  const i64 ist = l_nodalgrid ? 0 : 1;
#pragma omp parallel for schedule(static)
  for (i64 l = -nzs; l <= nz + nzs; ++l)
    for (i64 k = -nys; k <= ny + nys; ++k)
      for (i64 j = -nxs; j <= nx + nxs; ++j) {
        Ex(j, k, l) = Ex(j, k, l) - mudt * Jx(j, k, l);
        for (i64 i = 1; i <= nord_hi(nordery / 2, ny, nyguard, k); ++i)
          Ex(j, k, l) = Ex(j, k, l) + dtsdy[i - 1] * (Bz(j, k + i - ist, l) - Bz(j, k - i, l));
        for (i64 i = 1; i <= nord_hi(norderz / 2, nz, nzguard, l); ++i)
          Ex(j, k, l) = Ex(j, k, l) - dtsdz[i - 1] * (By(j, k, l + i - ist) - By(j, k, l - i));
      }
#pragma omp parallel for schedule(static)
  for (i64 l = -nzs; l <= nz + nzs; ++l)
    for (i64 k = -nys; k <= ny + nys; ++k)
      for (i64 j = -nxs; j <= nx + nxs; ++j) {
        Ey(j, k, l) = Ey(j, k, l) - mudt * Jy(j, k, l);
        for (i64 i = 1; i <= nord_hi(norderx / 2, nx, nxguard, j); ++i)
          Ey(j, k, l) = Ey(j, k, l) - dtsdx[i - 1] * (Bz(j + i - ist, k, l) - Bz(j - i, k, l));
        for (i64 i = 1; i <= nord_hi(norderz / 2, nz, nzguard, l); ++i)
          Ey(j, k, l) = Ey(j, k, l) + dtsdz[i - 1] * (Bx(j, k, l + i - ist) - Bx(j, k, l - i));
      }
#pragma omp parallel for schedule(static)
  for (i64 l = -nzs; l <= nz + nzs; ++l)
    for (i64 k = -nys; k <= ny + nys; ++k)
      for (i64 j = -nxs; j <= nx + nxs; ++j) {
        Ez(j, k, l) = Ez(j, k, l) - mudt * Jz(j, k, l);
        for (i64 i = 1; i <= nord_hi(norderx / 2, nx, nxguard, j); ++i)
          Ez(j, k, l) = Ez(j, k, l) + dtsdx[i - 1] * (By(j + i - ist, k, l) - By(j - i, k, l));
        for (i64 i = 1; i <= nord_hi(nordery / 2, ny, nyguard, k); ++i)
          Ez(j, k, l) = Ez(j, k, l) - dtsdy[i - 1] * (Bx(j, k + i - ist, l) - Bx(j, k - i, l));
      }
}

void orc_pxrpush_em3d_bvec_norder(double* ex_, double* ey_, double* ez_, double* bx_,
                                  double* by_, double* bz_, const double* dtsdx,
                                  const double* dtsdy, const double* dtsdz, i64 nx, i64 ny,
                                  i64 nz, i64 norderx, i64 nordery, i64 norderz, i64 nxguard,
                                  i64 nyguard, i64 nzguard, i64 nxs, i64 nys, i64 nzs,
                                  i64 l_nodalgrid) {
  F3 Ex = gview(ex_, nx, ny, nz, nxguard, nyguard, nzguard);
  F3 Ey = gview(ey_, nx, ny, nz, nxguard, nyguard, nzguard);
  F3 Ez = gview(ez_, nx, ny, nz, nxguard, nyguard, nzguard);
  F3 Bx = gview(bx_, nx, ny, nz, nxguard, nyguard, nzguard);
  F3 By = gview(by_, nx, ny, nz, nxguard, nyguard, nzguard);
  F3 Bz = gview(bz_, nx, ny, nz, nxguard, nyguard, nzguard);
  const i64 ist = l_nodalgrid ? 0 : 1;
#pragma omp parallel for schedule(static)
  for (i64 l = -nzs; l <= nz + nzs; ++l)
    for (i64 k = -nys; k <= ny + nys; ++k)
      for (i64 j = -nxs; j <= nx + nxs; ++j) {
        for (i64 i = 1; i <= nord_hi(nordery / 2, ny, nyguard, k); ++i)
          Bx(j, k, l) = Bx(j, k, l) - dtsdy[i - 1] * (Ez(j, k + i, l) - Ez(j, k - i + ist, l));
        for (i64 i = 1; i <= nord_hi(norderz / 2, nz, nzguard, l); ++i)
          Bx(j, k, l) = Bx(j, k, l) + dtsdz[i - 1] * (Ey(j, k, l + i) - Ey(j, k, l - i + ist));
      }
#pragma omp parallel for schedule(static)
  for (i64 l = -nzs; l <= nz + nzs; ++l)
    for (i64 k = -nys; k <= ny + nys; ++k)
      for (i64 j = -nxs; j <= nx + nxs; ++j) {
        for (i64 i = 1; i <= nord_hi(norderx / 2, nx, nxguard, j); ++i)
          By(j, k, l) = By(j, k, l) + dtsdx[i - 1] * (Ez(j + i, k, l) - Ez(j - i + ist, k, l));
        for (i64 i = 1; i <= nord_hi(norderz / 2, nz, nzguard, l); ++i)
          By(j, k, l) = By(j, k, l) - dtsdz[i - 1] * (Ex(j, k, l + i) - Ex(j, k, l - i + ist));
      }
#pragma omp parallel for schedule(static)
  for (i64 l = -nzs; l <= nz + nzs; ++l)
    for (i64 k = -nys; k <= ny + nys; ++k)
      for (i64 j = -nxs; j <= nx + nxs; ++j) {
        for (i64 i = 1; i <= nord_hi(norderx / 2, nx, nxguard, j); ++i)
          Bz(j, k, l) = Bz(j, k, l) - dtsdx[i - 1] * (Ey(j + i, k, l) - Ey(j - i + ist, k, l));
        for (i64 i = 1; i <= nord_hi(nordery / 2, ny, nyguard, k); ++i)
          Bz(j, k, l) = Bz(j, k, l) + dtsdy[i - 1] * (Ex(j, k + i, l) - Ex(j, k - i + ist, l));
      }
}

// particle_bcs for one domain with per-side pbound codes
// (particle_boundaries.F90:1098-1300): pb[6] = x-, x+, y-, y+, z-, z+;
// 0 periodic, 1 absorbing, 2 reflecting, 3 reinjecting (see the cases
// there); lo/hi: x_min_local_part ... (also xmin_part ... here), tlo/thi: the
// tile particle region for the reinjection clamps.  Removal as
// rm_particles_from_species_with_mask (tiling.F90:522-537): from the last
// particle down, a removed one is replaced by the current last one.  Arrays
// w and id may be NULL.  Returns the particle count left.
i64 orc_particle_bcs(i64 np, double* x, double* y, double* z, double* ux, double* uy,
                     double* uz, double* gi, double* w, double* id, const double* lo,
                     const double* hi, const double* d, const i64* pb, const double* tlo,
                     const double* thi) {
  std::vector<char> mask(np, 1);
  double* P[3] = {x, y, z};
  double* U[3] = {ux, uy, uz};
  for (i64 i = 0; i < np; ++i) {
    bool done = false;
    for (int a = 0; a < 3 && !done; ++a) {
      const double part_xyz = P[a][i];
      const double length = hi[a] - lo[a];
      if (part_xyz < lo[a]) {
        switch (pb[2 * a]) {
          case 1: mask[i] = 0; done = true; break;
          case 2: P[a][i] = part_xyz + d[a]; U[a][i] = -U[a][i]; break;
          case 3:
            P[a][i] = 2.0 * lo[a] - P[a][i];
            ux[i] = 0.; uy[i] = 0.; uz[i] = 0.;
            for (int b = 0; b < 3; ++b) {
              P[b][i] = std::max(P[b][i], tlo[b] + 0.5 * d[b]);
              P[b][i] = std::min(P[b][i], thi[b] - 0.5 * d[b]);
            }
            done = true;
            break;
          default: P[a][i] = part_xyz + length;
        }
      }
      if (done) break;
      if (part_xyz >= hi[a]) {
        switch (pb[2 * a + 1]) {
          case 1: mask[i] = 0; done = true; break;
          case 2: P[a][i] = part_xyz - d[a]; U[a][i] = -U[a][i]; break;
          case 3:
            P[a][i] = 2.0 * hi[a] - P[a][i];
            ux[i] = 0.; uy[i] = 0.; uz[i] = 0.;
            for (int b = 0; b < 3; ++b) {
              P[b][i] = std::max(P[b][i], tlo[b] + 0.5 * d[b]);
              P[b][i] = std::min(P[b][i], thi[b] - 0.5 * d[b]);
            }
            done = true;
            break;
          default: P[a][i] = part_xyz - length;
        }
      }
    }
  }
  double* cols[9] = {x, y, z, ux, uy, uz, gi, w, id};
  i64 n = np;
  for (i64 i = np - 1; i >= 0; --i) {
    if (mask[i]) continue;
    if (i != n - 1)
      for (double* c : cols)
        if (c) c[i] = c[n - 1];
    n = n - 1;
  }
  return n;
}

// FD_weights (submain.F90:927-984): Fornberg's recursion for the weights of
// the first derivative on norder+1 points x_i = i - n/2 + 1 at the point z
// (0.5 on the staggered grid, 0 on the nodal one); coeffs(i) = c(1, n/2+i-1).
void orc_FD_weights(double* coeffs, i64 norder, i64 l_nodal) {
  const double z = l_nodal ? 0.0 : 0.5;
  const i64 m = 1, n = norder + 1;
  std::vector<double> x(n), c((m + 1) * n, 0.0);
  auto C = [&](i64 k, i64 i) -> double& { return c[k + (m + 1) * i]; };
  for (i64 i = 0; i <= n - 1; ++i) x[i] = (double)(i - n / 2 + 1);
  double c1 = 1.0, c4 = x[0] - z;
  C(0, 0) = 1.0;
  for (i64 i = 1; i <= n - 1; ++i) {
    const i64 mn = std::min(i + 1, m + 1);
    double c2 = 1.0;
    const double c5 = c4;
    c4 = x[i] - z;
    for (i64 j = 0; j <= i - 1; ++j) {
      const double c3 = x[i] - x[j];
      c2 = c2 * c3;
      if (j == i - 1) {
        for (i64 k = 1; k <= mn - 1; ++k) C(k, i) = c1 * (k * C(k - 1, i - 1) - c5 * C(k, i - 1)) / c2;
        C(0, i) = -c1 * c5 * C(0, i - 1) / c2;
        for (i64 k = 1; k <= mn - 1; ++k) C(k, j) = (c4 * C(k, j) - k * C(k - 1, j)) / c3;
        C(0, j) = c4 * C(0, j) / c3;
      }
    }
    c1 = c2;
  }
  for (i64 i = 1; i <= norder / 2; ++i) coeffs[i - 1] = C(m, norder / 2 + i - 1);
}

void orc_pxrpush_em3d_evec(const i64* bnds, double* ex_, double* ey_, double* ez_,
                           double* bx_, double* by_, double* bz_, double* jx_,
                           double* jy_, double* jz_, const i64* alo, const i64* ahi,
                           double mudt, double dtsdx, double dtsdy, double dtsdz) {
  F3 Ex = bview(ex_, alo + 0, ahi + 0), Ey = bview(ey_, alo + 3, ahi + 3),
     Ez = bview(ez_, alo + 6, ahi + 6), Bx = bview(bx_, alo + 9, ahi + 9),
     By = bview(by_, alo + 12, ahi + 12), Bz = bview(bz_, alo + 15, ahi + 15),
     Jx = bview(jx_, alo + 18, ahi + 18), Jy = bview(jy_, alo + 21, ahi + 21),
     Jz = bview(jz_, alo + 24, ahi + 24);
  const i64 *xlo = bnds, *xhi = bnds + 3, *ylo = bnds + 6, *yhi = bnds + 9,
            *zlo = bnds + 12, *zhi = bnds + 15;
#pragma omp parallel for schedule(static)
  for (i64 l = xlo[2]; l <= xhi[2]; ++l)
    for (i64 k = xlo[1]; k <= xhi[1]; ++k)
      for (i64 j = xlo[0]; j <= xhi[0]; ++j)
        Ex(j, k, l) = Ex(j, k, l) + dtsdy * (Bz(j, k, l) - Bz(j, k - 1, l)) -
                      dtsdz * (By(j, k, l) - By(j, k, l - 1)) - mudt * Jx(j, k, l);
#pragma omp parallel for schedule(static)
  for (i64 l = ylo[2]; l <= yhi[2]; ++l)
    for (i64 k = ylo[1]; k <= yhi[1]; ++k)
      for (i64 j = ylo[0]; j <= yhi[0]; ++j)
        Ey(j, k, l) = Ey(j, k, l) - dtsdx * (Bz(j, k, l) - Bz(j - 1, k, l)) +
                      dtsdz * (Bx(j, k, l) - Bx(j, k, l - 1)) - mudt * Jy(j, k, l);
#pragma omp parallel for schedule(static)
  for (i64 l = zlo[2]; l <= zhi[2]; ++l)
    for (i64 k = zlo[1]; k <= zhi[1]; ++k)
      for (i64 j = zlo[0]; j <= zhi[0]; ++j)
        Ez(j, k, l) = Ez(j, k, l) + dtsdx * (By(j, k, l) - By(j - 1, k, l)) -
                      dtsdy * (Bx(j, k, l) - Bx(j, k - 1, l)) - mudt * Jz(j, k, l);
}

void orc_pxrpush_em3d_bvec(const i64* bnds, double* ex_, double* ey_, double* ez_,
                           double* bx_, double* by_, double* bz_, const i64* alo,
                           const i64* ahi, double dtsdx, double dtsdy, double dtsdz) {
  F3 Ex = bview(ex_, alo + 0, ahi + 0), Ey = bview(ey_, alo + 3, ahi + 3),
     Ez = bview(ez_, alo + 6, ahi + 6), Bx = bview(bx_, alo + 9, ahi + 9),
     By = bview(by_, alo + 12, ahi + 12), Bz = bview(bz_, alo + 15, ahi + 15);
  const i64 *xlo = bnds, *xhi = bnds + 3, *ylo = bnds + 6, *yhi = bnds + 9,
            *zlo = bnds + 12, *zhi = bnds + 15;
#pragma omp parallel for schedule(static)
  for (i64 l = xlo[2]; l <= xhi[2]; ++l)
    for (i64 k = xlo[1]; k <= xhi[1]; ++k)
      for (i64 j = xlo[0]; j <= xhi[0]; ++j)
        Bx(j, k, l) = Bx(j, k, l) - dtsdy * (Ez(j, k + 1, l) - Ez(j, k, l)) +
                      dtsdz * (Ey(j, k, l + 1) - Ey(j, k, l));
#pragma omp parallel for schedule(static)
  for (i64 l = ylo[2]; l <= yhi[2]; ++l)
    for (i64 k = ylo[1]; k <= yhi[1]; ++k)
      for (i64 j = ylo[0]; j <= yhi[0]; ++j)
        By(j, k, l) = By(j, k, l) + dtsdx * (Ez(j + 1, k, l) - Ez(j, k, l)) -
                      dtsdz * (Ex(j, k, l + 1) - Ex(j, k, l));
#pragma omp parallel for schedule(static)
  for (i64 l = zlo[2]; l <= zhi[2]; ++l)
    for (i64 k = zlo[1]; k <= zhi[1]; ++k)
      for (i64 j = zlo[0]; j <= zhi[0]; ++j)
        Bz(j, k, l) = Bz(j, k, l) - dtsdx * (Ey(j + 1, k, l) - Ey(j, k, l)) +
                      dtsdy * (Ex(j, k + 1, l) - Ex(j, k, l));
}

// ----------------------------------------------------------------------------
// Periodic single-domain boundary exchanges.
// field_bc -> exchange_mpi_3d_grid_array_with_guards with both neighbours
// equal to the rank itself (src/boundary_conditions/field_boundaries.F90:107-269):
// per axis x, y, z in turn, the (g+1)-thick slab [0, g] is copied into
// [n, n+g], then the (updated) slab [n-g, n] into [-g, 0]; each slab spans the
// full (guarded) extent of the other two axes, so edges and corners propagate.
// summation_bcs (:403-503): per axis, A[0:g] += A[n:n+g], then
// A[n-g:n] += A[-g:0], then field_bc.
// ----------------------------------------------------------------------------
static void slab_copy(F3& a, int axis, i64 src, i64 dst, i64 cnt, const i64* ext_lo,
                      const i64* ext_hi, bool add) {
  // MPI_SENDRECV packs the send slab before the receive is unpacked.
  i64 lo[3] = {ext_lo[0], ext_lo[1], ext_lo[2]}, hi[3] = {ext_hi[0], ext_hi[1], ext_hi[2]};
  lo[axis] = 0; hi[axis] = cnt - 1;
  std::vector<double> tmp;
  tmp.reserve((hi[0] - lo[0] + 1) * (hi[1] - lo[1] + 1) * (hi[2] - lo[2] + 1));
  for (i64 k = lo[2]; k <= hi[2]; ++k)
    for (i64 j = lo[1]; j <= hi[1]; ++j)
      for (i64 i = lo[0]; i <= hi[0]; ++i) {
        i64 c[3] = {i, j, k}; c[axis] += src;
        tmp.push_back(a(c[0], c[1], c[2]));
      }
  size_t n = 0;
  for (i64 k = lo[2]; k <= hi[2]; ++k)
    for (i64 j = lo[1]; j <= hi[1]; ++j)
      for (i64 i = lo[0]; i <= hi[0]; ++i) {
        i64 c[3] = {i, j, k}; c[axis] += dst;
        double& d = a(c[0], c[1], c[2]);
        d = add ? d + tmp[n] : tmp[n];
        ++n;
      }
}

void orc_field_bc_periodic(double* f, i64 nx, i64 ny, i64 nz, i64 nxg, i64 nyg, i64 nzg) {
  F3 a = gview(f, nx, ny, nz, nxg, nyg, nzg);
  const i64 n[3] = {nx, ny, nz}, g[3] = {nxg, nyg, nzg};
  const i64 elo[3] = {-nxg, -nyg, -nzg}, ehi[3] = {nx + nxg, ny + nyg, nz + nzg};
  for (int ax = 0; ax < 3; ++ax) {
    slab_copy(a, ax, 0, n[ax], g[ax] + 1, elo, ehi, false);
    slab_copy(a, ax, n[ax] - g[ax], -g[ax], g[ax] + 1, elo, ehi, false);
  }
}

void orc_summation_bcs_periodic(double* f, i64 nx, i64 ny, i64 nz, i64 nxg, i64 nyg,
                                i64 nzg) {
  F3 a = gview(f, nx, ny, nz, nxg, nyg, nzg);
  const i64 n[3] = {nx, ny, nz}, g[3] = {nxg, nyg, nzg};
  const i64 elo[3] = {-nxg, -nyg, -nzg}, ehi[3] = {nx + nxg, ny + nyg, nz + nzg};
  for (int ax = 0; ax < 3; ++ax) {
    slab_copy(a, ax, n[ax], 0, g[ax] + 1, elo, ehi, true);
    slab_copy(a, ax, -g[ax], n[ax] - g[ax], g[ax] + 1, elo, ehi, true);
  }
  orc_field_bc_periodic(f, nx, ny, nz, nxg, nyg, nzg);
}

// c_dim = 2 (x-z arrays, ny = 0, no y guards): the same exchanges along x and
// z only; the reference skips the y exchange there (field_boundaries.F90:330,
// :444).
void orc_field_bc_periodic_2d(double* f, i64 nx, i64 nz, i64 nxg, i64 nzg) {
  F3 a = gview(f, nx, 0, nz, nxg, 0, nzg);
  const i64 n[3] = {nx, 0, nz}, g[3] = {nxg, 0, nzg};
  const i64 elo[3] = {-nxg, 0, -nzg}, ehi[3] = {nx + nxg, 0, nz + nzg};
  for (int ax = 0; ax < 3; ax += 2) {
    slab_copy(a, ax, 0, n[ax], g[ax] + 1, elo, ehi, false);
    slab_copy(a, ax, n[ax] - g[ax], -g[ax], g[ax] + 1, elo, ehi, false);
  }
}

void orc_summation_bcs_periodic_2d(double* f, i64 nx, i64 nz, i64 nxg, i64 nzg) {
  F3 a = gview(f, nx, 0, nz, nxg, 0, nzg);
  const i64 n[3] = {nx, 0, nz}, g[3] = {nxg, 0, nzg};
  const i64 elo[3] = {-nxg, 0, -nzg}, ehi[3] = {nx + nxg, 0, nz + nzg};
  for (int ax = 0; ax < 3; ax += 2) {
    slab_copy(a, ax, n[ax], 0, g[ax] + 1, elo, ehi, true);
    slab_copy(a, ax, -g[ax], n[ax] - g[ax], g[ax] + 1, elo, ehi, true);
  }
  orc_field_bc_periodic_2d(f, nx, nz, nxg, nzg);
}

// ----------------------------------------------------------------------------
// Diagnostics.  src/diags/diags.F90:129-168 (calc_field_div),
// :1072-1114 (get_loc_field_energy: sum over 1..n of 0.5*F^2 times dV),
// :847-938 (get_loc_kinetic_energy: sum (1/gaminv - 1)*w),
// :1305-1358 (get_norm_divErho over 1..n).
// ----------------------------------------------------------------------------
void orc_calc_field_div(double* dive_, const double* ex_, const double* ey_,
                        const double* ez_, i64 nx, i64 ny, i64 nz, i64 nxg, i64 nyg,
                        i64 nzg, double dx, double dy, double dz) {
  F3 dv = gview(dive_, nx, ny, nz, nxg, nyg, nzg);
  F3 ex = gview(const_cast<double*>(ex_), nx, ny, nz, nxg, nyg, nzg);
  F3 ey = gview(const_cast<double*>(ey_), nx, ny, nz, nxg, nyg, nzg);
  F3 ez = gview(const_cast<double*>(ez_), nx, ny, nz, nxg, nyg, nzg);
  const double invdx = 1.0 / dx, invdy = 1.0 / dy, invdz = 1.0 / dz;
  for (i64 l = 0; l <= nz; ++l)
    for (i64 k = 0; k <= ny; ++k)
      for (i64 j = 0; j <= nx; ++j)
        dv(j, k, l) = invdx * (ex(j, k, l) - ex(j - 1, k, l)) +
                      invdy * (ey(j, k, l) - ey(j, k - 1, l)) +
                      invdz * (ez(j, k, l) - ez(j, k, l - 1));
}

double orc_field_energy(const double* f_, i64 nx, i64 ny, i64 nz, i64 nxg, i64 nyg,
                        i64 nzg, double dx, double dy, double dz) {
  F3 f = gview(const_cast<double*>(f_), nx, ny, nz, nxg, nyg, nzg);
  double e = 0;
  for (i64 l = 1; l <= nz; ++l)
    for (i64 k = 1; k <= ny; ++k)
      for (i64 j = 1; j <= nx; ++j) e = e + f(j, k, l) * f(j, k, l) * 0.5;
  return e * dx * dy * dz;
}

double orc_kinetic_energy(i64 np, const double* gaminv, const double* w) {
  double e = 0;
  for (i64 ip = 0; ip < np; ++ip) {
    double partgam = 1.0 / gaminv[ip];
    e = e + (partgam - 1.0) * w[ip];
  }
  return e;
}

double orc_norm_diverho(const double* dive_, const double* rho_, i64 nx, i64 ny, i64 nz,
                        i64 nxg, i64 nyg, i64 nzg, double eps0) {
  F3 dv = gview(const_cast<double*>(dive_), nx, ny, nz, nxg, nyg, nzg);
  F3 rho = gview(const_cast<double*>(rho_), nx, ny, nz, nxg, nyg, nzg);
  double s = 0;
  for (i64 l = 1; l <= nz; ++l)
    for (i64 k = 1; k <= ny; ++k)
      for (i64 j = 1; j <= nx; ++j) s = s + sq(dv(j, k, l) * eps0 - rho(j, k, l));
  return std::sqrt(s);
}

}  // extern "C"

// ============================================================================
// Mini-app: tile geometry, tile drivers and the PIC step in the order of
// src/submain.F90:104-195 (3D branch, Yee solver, l_plasma):
//   field_gathering_plus_particle_pusher -> particle_bcs -> pxr_particle_sorting
//   -> pxrdepose_currents_on_grid_jxjyjz -> current_bcs -> push_bfield(dt/2)
//   -> bfield_bcs -> push_efield(dt) -> efield_bcs -> push_bfield(dt/2)
//   -> bfield_bcs -> calc_diags (rho deposit + charge_bcs).
// Single species, periodic single domain.  Every particle carries an id so
// results can be matched to other implementations after re-binning.
// ============================================================================
namespace {
struct OTile {
  i64 nmin[3], nmax[3];   // nx_tile_min/max (global node indices)
  i64 nc[3];              // nx_cells_tile
  i64 ng[3];              // nxg_tile
  double gmin[3];         // x_grid_tile_min
  double pmin[3], pmax[3];  // x_tile_min / x_tile_max (particle region)
  std::vector<double> x, y, z, ux, uy, uz, gi, ex, ey, ez, bx, by, bz, w, id;
  std::vector<double> a1, a2, a3;  // tile current arrays (-ng:nc+ng)
  i64 np() const { return (i64)x.size(); }
  void push_back(double px, double py, double pz, double pux, double puy, double puz,
                 double pg, double pw, double pid) {
    x.push_back(px); y.push_back(py); z.push_back(pz);
    ux.push_back(pux); uy.push_back(puy); uz.push_back(puz); gi.push_back(pg);
    ex.push_back(0); ey.push_back(0); ez.push_back(0);
    bx.push_back(0); by.push_back(0); bz.push_back(0);
    w.push_back(pw); id.push_back(pid);
  }
  // rm_particle_at_tile: the last particle takes the removed slot.
  void remove(i64 i) {
    i64 last = np() - 1;
    std::vector<double>* cols[] = {&x, &y, &z, &ux, &uy, &uz, &gi, &ex, &ey, &ez,
                                   &bx, &by, &bz, &w, &id};
    for (auto* c : cols) { (*c)[i] = (*c)[last]; c->pop_back(); }
  }
};

struct OSim {
  i64 n[3];             // cells
  i64 g;                // guard cells (fields and currents)
  double d[3], lo[3], hi[3];
  double dt, q, m, clight, mu0, eps0;
  i64 order, pusher, nt[3], lvect, sorting_period, it;
  i64 n0[3];            // nodes per tile (nx0_grid_tile)
  std::vector<double> ex, ey, ez, bx, by, bz, jx, jy, jz, rho, dive;
  std::vector<OTile> tiles;
  i64 gsize() const { return (n[0] + 1 + 2 * g) * (n[1] + 1 + 2 * g) * (n[2] + 1 + 2 * g); }
  OTile& tile(i64 ix, i64 iy, i64 iz) { return tiles[ix + nt[0] * (iy + nt[1] * iz)]; }
  F3 view(std::vector<double>& a) { return gview(a.data(), n[0], n[1], n[2], g, g, g); }
};

// set_tile_split_for_species (tiling.F90:94-261) and the guard choice of
// init_tile_arrays_for_species (:762-776).
void tile_split(OSim& s) {
  for (int ax = 0; ax < 3; ++ax) {
    i64 ngrid = s.n[ax] + 1;
    s.n0[ax] = ngrid / s.nt[ax];
    if (s.n0[ax] < 4) { s.nt[ax] = 1; s.n0[ax] = ngrid; }
  }
  s.tiles.assign(s.nt[0] * s.nt[1] * s.nt[2], OTile());
  for (i64 iz = 0; iz < s.nt[2]; ++iz)
    for (i64 iy = 0; iy < s.nt[1]; ++iy)
      for (i64 ix = 0; ix < s.nt[0]; ++ix) {
        OTile& t = s.tile(ix, iy, iz);
        i64 idx[3] = {ix, iy, iz};
        for (int ax = 0; ax < 3; ++ax) {
          i64 i = idx[ax], ntx = s.nt[ax], n0 = s.n0[ax];
          i64 ngrid = s.n[ax] + 1;
          i64 n0last = n0 + (ngrid - n0 * ntx);
          double dx = s.d[ax];
          if (i == 0) {
            t.nc[ax] = n0 - 1;
            t.gmin[ax] = s.lo[ax];
            double gmax = t.gmin[ax] + (n0 - 1) * dx;
            t.pmin[ax] = t.gmin[ax];
            t.pmax[ax] = gmax + dx / 2.0;
            t.nmin[ax] = 0;
          }
          if (i > 0 && i < ntx - 1) {
            t.nc[ax] = n0 - 1;
            t.gmin[ax] = s.lo[ax] + i * n0 * dx;
            double gmax = t.gmin[ax] + t.nc[ax] * dx;
            t.nmin[ax] = i * n0;
            t.pmin[ax] = t.gmin[ax] - dx / 2.0;
            t.pmax[ax] = gmax + dx / 2.0;
          }
          if (i == ntx - 1) {
            t.nc[ax] = n0last - 1;
            t.gmin[ax] = s.lo[ax] + i * n0 * dx;
            t.nmin[ax] = i * n0;
            t.pmin[ax] = t.gmin[ax] - dx / 2.0;
            t.pmax[ax] = s.hi[ax];
          }
          t.nmax[ax] = t.nmin[ax] + t.nc[ax];
          t.ng[ax] = (i > 0 && i < ntx - 1) ? std::max<i64>(s.order + 1, 2) : s.g;
        }
        size_t sz = (t.nc[0] + 1 + 2 * t.ng[0]) * (t.nc[1] + 1 + 2 * t.ng[1]) *
                    (t.nc[2] + 1 + 2 * t.ng[2]);
        t.a1.assign(sz, 0.0); t.a2.assign(sz, 0.0); t.a3.assign(sz, 0.0);
      }
}

// Tile index of a particle (particle_boundaries.F90:428-535), 0-based.
inline i64 tile_index(const OSim& s, int ax, double x) {
  i64 ind = ffloor((x - s.lo[ax] + s.d[ax] / 2.0) / (s.n0[ax] * s.d[ax]));
  return std::min<i64>(ind, s.nt[ax] - 1);
}

void gather_push_tiles(OSim& s) {
  const i64 ntiles = (i64)s.tiles.size();
#pragma omp parallel for schedule(dynamic)
  for (i64 t = 0; t < ntiles; ++t) {
    OTile& tl = s.tiles[t];
    i64 np = tl.np();
    if (np == 0) continue;
    // extile = exg(jmin:jmax, kmin:kmax, lmin:lmax), guard = tile guard
    i64 lo[3], hi[3], ext[3];
    for (int ax = 0; ax < 3; ++ax) {
      lo[ax] = tl.nmin[ax] - tl.ng[ax]; hi[ax] = tl.nmax[ax] + tl.ng[ax];
      ext[ax] = hi[ax] - lo[ax] + 1;
    }
    size_t sz = ext[0] * ext[1] * ext[2];
    std::vector<double> T[6];
    std::vector<double>* G[6] = {&s.ex, &s.ey, &s.ez, &s.bx, &s.by, &s.bz};
    for (int c = 0; c < 6; ++c) {
      T[c].resize(sz);
      F3 gv = s.view(*G[c]);
      size_t n = 0;
      for (i64 l = lo[2]; l <= hi[2]; ++l)
        for (i64 k = lo[1]; k <= hi[1]; ++k)
          for (i64 j = lo[0]; j <= hi[0]; ++j) T[c][n++] = gv(j, k, l);
    }
    std::fill(tl.ex.begin(), tl.ex.end(), 0.0); std::fill(tl.ey.begin(), tl.ey.end(), 0.0);
    std::fill(tl.ez.begin(), tl.ez.end(), 0.0); std::fill(tl.bx.begin(), tl.bx.end(), 0.0);
    std::fill(tl.by.begin(), tl.by.end(), 0.0); std::fill(tl.bz.begin(), tl.bz.end(), 0.0);
    auto fn = s.order == 1 ? orc_field_gathering_plus_particle_pusher_1_1_1
            : s.order == 2 ? orc_field_gathering_plus_particle_pusher_2_2_2
                           : orc_field_gathering_plus_particle_pusher_3_3_3;
    fn(np, tl.x.data(), tl.y.data(), tl.z.data(), tl.ux.data(), tl.uy.data(), tl.uz.data(),
       tl.gi.data(), tl.ex.data(), tl.ey.data(), tl.ez.data(), tl.bx.data(), tl.by.data(),
       tl.bz.data(), tl.gmin[0], tl.gmin[1], tl.gmin[2], s.d[0], s.d[1], s.d[2], tl.nc[0],
       tl.nc[1], tl.nc[2], tl.ng[0], tl.ng[1], tl.ng[2], T[0].data(), T[1].data(),
       T[2].data(), T[3].data(), T[4].data(), T[5].data(), s.q, s.m, s.lvect, s.dt,
       s.pusher, s.clight);
  }
}

// Periodic wrap (particle_boundaries.F90:1109-1300, pbound = 0) followed by
// tile re-binning (particle_bcs_tiles, :428-535).
void particle_bcs(OSim& s) {
  const i64 ntiles = (i64)s.tiles.size();
  double len[3] = {s.hi[0] - s.lo[0], s.hi[1] - s.lo[1], s.hi[2] - s.lo[2]};
  for (i64 t = 0; t < ntiles; ++t) {
    OTile& tl = s.tiles[t];
    std::vector<double>* P[3] = {&tl.x, &tl.y, &tl.z};
    for (i64 i = 0; i < tl.np(); ++i)
      for (int ax = 0; ax < 3; ++ax) {
        double& v = (*P[ax])[i];
        if (v < s.lo[ax]) v = v + len[ax];
        else if (v >= s.hi[ax]) v = v - len[ax];
      }
  }
  for (i64 t = 0; t < ntiles; ++t) {
    OTile& tl = s.tiles[t];
    for (i64 i = tl.np() - 1; i >= 0; --i) {
      double p[3] = {tl.x[i], tl.y[i], tl.z[i]};
      bool inside = true;
      for (int ax = 0; ax < 3; ++ax)
        inside = inside && (p[ax] >= tl.pmin[ax]) && (p[ax] < tl.pmax[ax]);
      if (inside) continue;
      i64 ix = tile_index(s, 0, p[0]), iy = tile_index(s, 1, p[1]), iz = tile_index(s, 2, p[2]);
      OTile& dst = s.tile(ix, iy, iz);
      if (&dst == &tl) continue;
      dst.push_back(tl.x[i], tl.y[i], tl.z[i], tl.ux[i], tl.uy[i], tl.uz[i], tl.gi[i],
                    tl.w[i], tl.id[i]);
      tl.remove(i);
    }
  }
}

// pxr_particle_bin_sorting (sorting.F90:247-361): stable counting sort of each
// tile by cell bin, with bins of size sorting_dx = dx starting at x_tile_min.
void sort_tiles(OSim& s) {
  for (OTile& tl : s.tiles) {
    i64 np = tl.np();
    if (np == 0) continue;
    double xmn[3], xmx[3];
    i64 nb[3];
    for (int ax = 0; ax < 3; ++ax) {
      xmn[ax] = tl.pmin[ax]; xmx[ax] = tl.pmax[ax] + s.d[ax];
      nb[ax] = (i64)std::ceil((xmx[ax] - xmn[ax]) * (1.0 / s.d[ax]));
    }
    i64 nbhc = nb[0] * nb[1] * nb[2];
    std::vector<i64> hc(np), cnt(nbhc + 1, 0);
    for (i64 ip = 0; ip < np; ++ip) {
      i64 ix = ffloor((tl.x[ip] - xmn[0]) * (1.0 / s.d[0]));
      i64 iy = ffloor((tl.y[ip] - xmn[1]) * (1.0 / s.d[1]));
      i64 iz = ffloor((tl.z[ip] - xmn[2]) * (1.0 / s.d[2]));
      hc[ip] = iz * nb[0] * nb[1] + iy * nb[0] + ix;
      if (hc[ip] < 0 || hc[ip] >= nbhc) hc[ip] = std::min(std::max<i64>(hc[ip], 0), nbhc - 1);
      cnt[hc[ip] + 1]++;
    }
    for (i64 c = 0; c < nbhc; ++c) cnt[c + 1] += cnt[c];
    std::vector<i64> perm(np);
    for (i64 ip = 0; ip < np; ++ip) perm[cnt[hc[ip]]++] = ip;
    std::vector<double>* cols[] = {&tl.x, &tl.y, &tl.z, &tl.ux, &tl.uy, &tl.uz, &tl.gi,
                                   &tl.w, &tl.id};
    for (auto* c : cols) {
      std::vector<double> tmp(np);
      for (i64 k = 0; k < np; ++k) tmp[k] = (*c)[perm[k]];
      c->swap(tmp);
    }
  }
}

// pxrdepose_currents_on_grid_jxjyjz_esirkepov_sub_openmp
// (current_deposition_manager_3d.F90:1534-1813): deposit per tile into the
// tile arrays, add the tile interior, then the +-x, +-y, +-z guard faces.
void deposit_tiles(OSim& s) {
  std::fill(s.jx.begin(), s.jx.end(), 0.0);
  std::fill(s.jy.begin(), s.jy.end(), 0.0);
  std::fill(s.jz.begin(), s.jz.end(), 0.0);
  const i64 ntiles = (i64)s.tiles.size();
#pragma omp parallel for schedule(dynamic)
  for (i64 t = 0; t < ntiles; ++t) {
    OTile& tl = s.tiles[t];
    std::fill(tl.a1.begin(), tl.a1.end(), 0.0);
    std::fill(tl.a2.begin(), tl.a2.end(), 0.0);
    std::fill(tl.a3.begin(), tl.a3.end(), 0.0);
    if (tl.np() == 0) continue;
    orc_depose_jxjyjz(tl.a1.data(), tl.a2.data(), tl.a3.data(), tl.np(), tl.x.data(),
                      tl.y.data(), tl.z.data(), tl.ux.data(), tl.uy.data(), tl.uz.data(),
                      tl.gi.data(), tl.w.data(), s.q, tl.gmin[0], tl.gmin[1], tl.gmin[2],
                      s.dt, s.d[0], s.d[1], s.d[2], tl.nc[0], tl.nc[1], tl.nc[2], tl.ng[0],
                      tl.ng[1], tl.ng[2], s.order, s.order, s.order, 0, s.clight);
  }
  F3 J[3] = {s.view(s.jx), s.view(s.jy), s.view(s.jz)};
  // phase 1: interiors (disjoint between tiles)
#pragma omp parallel for schedule(dynamic)
  for (i64 t = 0; t < ntiles; ++t) {
    OTile& tl = s.tiles[t];
    if (tl.np() == 0) continue;
    std::vector<double>* A[3] = {&tl.a1, &tl.a2, &tl.a3};
    for (int c = 0; c < 3; ++c) {
      F3 a = gview(A[c]->data(), tl.nc[0], tl.nc[1], tl.nc[2], tl.ng[0], tl.ng[1], tl.ng[2]);
      for (i64 l = 0; l <= tl.nc[2]; ++l)
        for (i64 k = 0; k <= tl.nc[1]; ++k)
          for (i64 j = 0; j <= tl.nc[0]; ++j) {
            double& d = J[c](tl.nmin[0] + j, tl.nmin[1] + k, tl.nmin[2] + l);
            d = d + a(j, k, l);
          }
    }
  }
  // phases 2-4: guard faces along x (full y,z guard span), then y (interior x),
  // then z (interior x,y)
  for (int ph = 0; ph < 3; ++ph) {
    for (i64 t = 0; t < ntiles; ++t) {
      OTile& tl = s.tiles[t];
      if (tl.np() == 0) continue;
      std::vector<double>* A[3] = {&tl.a1, &tl.a2, &tl.a3};
      for (int c = 0; c < 3; ++c) {
        F3 a = gview(A[c]->data(), tl.nc[0], tl.nc[1], tl.nc[2], tl.ng[0], tl.ng[1], tl.ng[2]);
        for (int side = 0; side < 2; ++side) {
          i64 lo[3], hi[3];
          for (int ax = 0; ax < 3; ++ax) {
            if (ax == ph) {
              lo[ax] = side == 0 ? -tl.ng[ax] : tl.nc[ax] + 1;
              hi[ax] = side == 0 ? -1 : tl.nc[ax] + tl.ng[ax];
            } else if (ax > ph) {
              lo[ax] = -tl.ng[ax]; hi[ax] = tl.nc[ax] + tl.ng[ax];
            } else {
              lo[ax] = 0; hi[ax] = tl.nc[ax];
            }
          }
          for (i64 l = lo[2]; l <= hi[2]; ++l)
            for (i64 k = lo[1]; k <= hi[1]; ++k)
              for (i64 j = lo[0]; j <= hi[0]; ++j) {
                double& d = J[c](tl.nmin[0] + j, tl.nmin[1] + k, tl.nmin[2] + l);
                d = d + a(j, k, l);
              }
        }
      }
    }
  }
}

void push_b(OSim& s, double frac) {
  i64 bnds[18], alo[18], ahi[18];
  for (int c = 0; c < 3; ++c)
    for (int ax = 0; ax < 3; ++ax) { bnds[6 * c + ax] = 0; bnds[6 * c + 3 + ax] = s.n[ax]; }
  for (int a = 0; a < 6; ++a)
    for (int ax = 0; ax < 3; ++ax) { alo[3 * a + ax] = -s.g; ahi[3 * a + ax] = s.n[ax] + s.g; }
  orc_pxrpush_em3d_bvec(bnds, s.ex.data(), s.ey.data(), s.ez.data(), s.bx.data(), s.by.data(),
                        s.bz.data(), alo, ahi, frac * s.dt / s.d[0], frac * s.dt / s.d[1],
                        frac * s.dt / s.d[2]);
}

void push_e(OSim& s) {
  i64 bnds[18], alo[27], ahi[27];
  for (int c = 0; c < 3; ++c)
    for (int ax = 0; ax < 3; ++ax) { bnds[6 * c + ax] = 0; bnds[6 * c + 3 + ax] = s.n[ax]; }
  for (int a = 0; a < 9; ++a)
    for (int ax = 0; ax < 3; ++ax) { alo[3 * a + ax] = -s.g; ahi[3 * a + ax] = s.n[ax] + s.g; }
  const double c2 = s.clight * s.clight;
  orc_pxrpush_em3d_evec(bnds, s.ex.data(), s.ey.data(), s.ez.data(), s.bx.data(), s.by.data(),
                        s.bz.data(), s.jx.data(), s.jy.data(), s.jz.data(), alo, ahi,
                        c2 * s.mu0 * s.dt, c2 * s.dt / s.d[0], c2 * s.dt / s.d[1],
                        c2 * s.dt / s.d[2]);
}

void bc3(OSim& s, std::vector<double>& a, std::vector<double>& b, std::vector<double>& c) {
  orc_field_bc_periodic(a.data(), s.n[0], s.n[1], s.n[2], s.g, s.g, s.g);
  orc_field_bc_periodic(b.data(), s.n[0], s.n[1], s.n[2], s.g, s.g, s.g);
  orc_field_bc_periodic(c.data(), s.n[0], s.n[1], s.n[2], s.g, s.g, s.g);
}

void deposit_rho(OSim& s) {
  std::fill(s.rho.begin(), s.rho.end(), 0.0);
  for (OTile& tl : s.tiles) {
    if (tl.np() == 0) continue;
    orc_depose_rho_scalar(s.order, s.rho.data(), tl.np(), tl.x.data(), tl.y.data(),
                          tl.z.data(), tl.w.data(), s.q, s.lo[0], s.lo[1], s.lo[2], s.d[0],
                          s.d[1], s.d[2], s.n[0], s.n[1], s.n[2], s.g, s.g, s.g);
  }
  orc_summation_bcs_periodic(s.rho.data(), s.n[0], s.n[1], s.n[2], s.g, s.g, s.g);
}
}  // namespace

extern "C" {

void* orc_sim_new(i64 nx, i64 ny, i64 nz, i64 g, double dx, double dy, double dz,
                  double xmin, double ymin, double zmin, double dt, double q, double m,
                  double clight, double mu0, double eps0, i64 order, i64 pusher,
                  i64 ntx, i64 nty, i64 ntz, i64 lvect, i64 sorting_period) {
  OSim* s = new OSim();
  s->n[0] = nx; s->n[1] = ny; s->n[2] = nz; s->g = g;
  s->d[0] = dx; s->d[1] = dy; s->d[2] = dz;
  s->lo[0] = xmin; s->lo[1] = ymin; s->lo[2] = zmin;
  s->hi[0] = xmin + nx * dx; s->hi[1] = ymin + ny * dy; s->hi[2] = zmin + nz * dz;
  s->dt = dt; s->q = q; s->m = m; s->clight = clight; s->mu0 = mu0; s->eps0 = eps0;
  s->order = order; s->pusher = pusher;
  s->nt[0] = ntx; s->nt[1] = nty; s->nt[2] = ntz;
  s->lvect = lvect; s->sorting_period = sorting_period; s->it = 0;
  i64 gs = s->gsize();
  for (auto* v : {&s->ex, &s->ey, &s->ez, &s->bx, &s->by, &s->bz, &s->jx, &s->jy, &s->jz,
                  &s->rho, &s->dive})
    v->assign(gs, 0.0);
  tile_split(*s);
  return s;
}

void orc_sim_free(void* h) { delete (OSim*)h; }

i64 orc_sim_grid_size(void* h) { return ((OSim*)h)->gsize(); }

// which: 0..5 ex..bz, 6..8 jx..jz, 9 rho, 10 dive.  dir 0: copy in, 1: out.
void orc_sim_field(void* h, i64 which, double* buf, i64 dir) {
  OSim* s = (OSim*)h;
  std::vector<double>* F[] = {&s->ex, &s->ey, &s->ez, &s->bx, &s->by, &s->bz,
                              &s->jx, &s->jy, &s->jz, &s->rho, &s->dive};
  std::vector<double>& v = *F[which];
  if (dir == 0) std::memcpy(v.data(), buf, v.size() * sizeof(double));
  else std::memcpy(buf, v.data(), v.size() * sizeof(double));
}

// Adds particles (gaminv computed as in pxr_set_gamma) to their tiles.
void orc_sim_add_particles(void* h, i64 np, const double* x, const double* y,
                           const double* z, const double* ux, const double* uy,
                           const double* uz, const double* w, const double* id) {
  OSim* s = (OSim*)h;
  const double clghtisq = 1.0 / sq(s->clight);
  for (i64 i = 0; i < np; ++i) {
    i64 ix = tile_index(*s, 0, x[i]), iy = tile_index(*s, 1, y[i]), iz = tile_index(*s, 2, z[i]);
    double usq = (sq(ux[i]) + sq(uy[i]) + sq(uz[i])) * clghtisq;
    s->tile(ix, iy, iz).push_back(x[i], y[i], z[i], ux[i], uy[i], uz[i],
                                  1.0 / std::sqrt(1.0 + usq), w[i], id[i]);
  }
}

i64 orc_sim_np(void* h) {
  OSim* s = (OSim*)h;
  i64 n = 0;
  for (auto& t : s->tiles) n += t.np();
  return n;
}

// Copies all particles out in tile order.  cols: x y z ux uy uz gaminv
// ex ey ez bx by bz w id (15 arrays of np each, contiguous: out[c*np + i]).
void orc_sim_get_particles(void* h, double* out) {
  OSim* s = (OSim*)h;
  i64 np = orc_sim_np(h), k = 0;
  for (auto& t : s->tiles) {
    const std::vector<double>* cols[] = {&t.x, &t.y, &t.z, &t.ux, &t.uy, &t.uz, &t.gi,
                                         &t.ex, &t.ey, &t.ez, &t.bx, &t.by, &t.bz, &t.w, &t.id};
    for (i64 i = 0; i < t.np(); ++i, ++k)
      for (int c = 0; c < 15; ++c) out[c * np + k] = (*cols[c])[i];
  }
}

// Copies selected particle columns out in tile order: cols[i] indexes the
// column list of orc_sim_get_particles; out[i*np + k].
void orc_sim_get_particle_columns(void* h, const i64* cols, i64 ncols, double* out) {
  OSim* s = (OSim*)h;
  const i64 np = orc_sim_np(h);
  for (i64 c = 0; c < ncols; ++c) {
    i64 k = 0;
    for (auto& t : s->tiles) {
      const std::vector<double>* all[] = {&t.x, &t.y, &t.z, &t.ux, &t.uy, &t.uz, &t.gi,
                                          &t.ex, &t.ey, &t.ez, &t.bx, &t.by, &t.bz, &t.w,
                                          &t.id};
      const std::vector<double>& v = *all[cols[c]];
      std::copy(v.begin(), v.end(), out + c * np + k);
      k += t.np();
    }
  }
}

// Runs nsteps PIC steps.  diag != 0: deposit rho and compute div E after each step.
void orc_sim_step(void* h, i64 nsteps, i64 diag) {
  OSim* s = (OSim*)h;
  for (i64 st = 0; st < nsteps; ++st) {
    gather_push_tiles(*s);
    particle_bcs(*s);
    if (s->sorting_period > 0 && (s->it % s->sorting_period) == 0) sort_tiles(*s);
    deposit_tiles(*s);
    orc_summation_bcs_periodic(s->jx.data(), s->n[0], s->n[1], s->n[2], s->g, s->g, s->g);
    orc_summation_bcs_periodic(s->jy.data(), s->n[0], s->n[1], s->n[2], s->g, s->g, s->g);
    orc_summation_bcs_periodic(s->jz.data(), s->n[0], s->n[1], s->n[2], s->g, s->g, s->g);
    push_b(*s, 0.5);
    bc3(*s, s->bx, s->by, s->bz);
    push_e(*s);
    bc3(*s, s->ex, s->ey, s->ez);
    push_b(*s, 0.5);
    bc3(*s, s->bx, s->by, s->bz);
    if (diag) {
      deposit_rho(*s);
      orc_calc_field_div(s->dive.data(), s->ex.data(), s->ey.data(), s->ez.data(), s->n[0],
                         s->n[1], s->n[2], s->g, s->g, s->g, s->d[0], s->d[1], s->d[2]);
    }
    s->it += 1;
  }
}

// Diagnostics of the current state: out[0] kinetic (sum (gamma-1) w m c^2),
// out[1..3] Ex,Ey,Ez energies (x eps0), out[4..6] Bx,By,Bz (/ mu0),
// out[7] ||div E * eps0 - rho||_2 (rho must be current: deposit_rho first).
void orc_sim_diags(void* h, double* out) {
  OSim* s = (OSim*)h;
  double ke = 0;
  for (auto& t : s->tiles) ke += orc_kinetic_energy(t.np(), t.gi.data(), t.w.data());
  out[0] = ke * s->m * s->clight * s->clight;
  std::vector<double>* F[] = {&s->ex, &s->ey, &s->ez, &s->bx, &s->by, &s->bz};
  for (int c = 0; c < 6; ++c) {
    double e = orc_field_energy(F[c]->data(), s->n[0], s->n[1], s->n[2], s->g, s->g, s->g,
                                s->d[0], s->d[1], s->d[2]);
    out[1 + c] = c < 3 ? e * s->eps0 : e / s->mu0;
  }
  deposit_rho(*s);
  orc_calc_field_div(s->dive.data(), s->ex.data(), s->ey.data(), s->ez.data(), s->n[0],
                     s->n[1], s->n[2], s->g, s->g, s->g, s->d[0], s->d[1], s->d[2]);
  out[7] = orc_norm_diverho(s->dive.data(), s->rho.data(), s->n[0], s->n[1], s->n[2], s->g,
                            s->g, s->g, s->eps0);
}

// Individual phases, exposed for fine-grained parity checks.
void orc_sim_phase(void* h, i64 phase) {
  OSim* s = (OSim*)h;
  switch (phase) {
    case 0: gather_push_tiles(*s); break;
    case 1: particle_bcs(*s); break;
    case 2: sort_tiles(*s); break;
    case 3: deposit_tiles(*s); break;
    case 4:
      orc_summation_bcs_periodic(s->jx.data(), s->n[0], s->n[1], s->n[2], s->g, s->g, s->g);
      orc_summation_bcs_periodic(s->jy.data(), s->n[0], s->n[1], s->n[2], s->g, s->g, s->g);
      orc_summation_bcs_periodic(s->jz.data(), s->n[0], s->n[1], s->n[2], s->g, s->g, s->g);
      break;
    case 5: push_b(*s, 0.5); bc3(*s, s->bx, s->by, s->bz); break;
    case 6: push_e(*s); bc3(*s, s->ex, s->ey, s->ez); break;
    case 7: deposit_rho(*s); break;
  }
}

int orc_num_threads() {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

}  // extern "C"
