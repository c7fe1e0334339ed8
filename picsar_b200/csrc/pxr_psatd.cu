// PSATD field push in Fourier space (the spectral solver of one periodic
// domain with a local FFT): the per-mode update of push_psaotd_ebfielfs_3d
// (src/field_solvers/Maxwell/GPSTD_solver/fourier_psaotd.F90:1538-1643) with
// the coefficient blocks of compute_cc_mat_merged_fields
// (src/field_solvers/Maxwell/GPSTD_solver/init_kspace_3D.F90:1316-1495) and
// the 1/(nfftx nffty nfftz) scaling of init_gpstd (:1025-1040).
//
// The reference keeps 33 complex coefficient blocks per mode.  Here each
// mode reads its three real operators at_op(1..3) and the separable k-vectors
// (forward and backward, per axis) and forms the entries it needs, so a mode
// moves 11 complex inputs, 3 reals and 6 complex outputs.  Summation order per
// output follows the reference (B from the old E, then E from the old B).
// Complex arrays are interleaved (re, im) FP64, modes x fastest.
#include "pxr_common.cuh"

namespace {

struct C2 {
  double r, i;
};

__device__ __forceinline__ C2 ld(const double* p, i64 m) { return C2{p[2 * m], p[2 * m + 1]}; }
__device__ __forceinline__ void st(double* p, i64 m, C2 v) {
  p[2 * m] = v.r;
  p[2 * m + 1] = v.i;
}
__device__ __forceinline__ C2 mul(C2 a, C2 b) {
  return C2{a.r * b.r - a.i * b.i, a.r * b.i + a.i * b.r};
}
__device__ __forceinline__ C2 add(C2 a, C2 b) { return C2{a.r + b.r, a.i + b.i}; }
__device__ __forceinline__ C2 scl(double s, C2 a) { return C2{s * a.r, s * a.i}; }
// i * k
__device__ __forceinline__ C2 ik(C2 k) { return C2{-k.i, k.r}; }

struct PsatdArgs {
  i64 nkx, nky, nkz;
  double *ex, *ey, *ez, *bx, *by, *bz;
  const double *jx, *jy, *jz, *rho, *rhoold;
  const double *kxf, *kxb, *kyf, *kyb, *kzf, *kzb;
  const double *kxc2, *kyc2, *kzc2;
  const double *at1, *at2, *at3;
  double c, eps0, mu0, dt, norm;
};

__global__ void k_psatd_push(PsatdArgs a) {
  const i64 nm = a.nkx * a.nky * a.nkz;
  for (i64 m = blockIdx.x * (i64)blockDim.x + threadIdx.x; m < nm;
       m += (i64)gridDim.x * blockDim.x) {
    const i64 ix = m % a.nkx, iy = (m / a.nkx) % a.nky, iz = m / (a.nkx * a.nky);
    const C2 Kxf = ld(a.kxf, ix), Kxb = ld(a.kxb, ix);
    const C2 Kyf = ld(a.kyf, iy), Kyb = ld(a.kyb, iy);
    const C2 Kzf = ld(a.kzf, iz), Kzb = ld(a.kzb, iz);
    const double c = a.c, n = a.norm;
    const double at1 = a.at1[m], at2 = a.at2[m], at3 = a.at3[m];
    const C2 ex = ld(a.ex, m), ey = ld(a.ey, m), ez = ld(a.ez, m);
    const C2 bx = ld(a.bx, m), by = ld(a.by, m), bz = ld(a.bz, m);
    const C2 jx = ld(a.jx, m), jy = ld(a.jy, m), jz = ld(a.jz, m);
    const C2 rh = ld(a.rho, m), ro = ld(a.rhoold, m);
    // coefficient blocks (already scaled by the FFT normalisation)
    const double d = at2 * n;                   // (i, i)
    const double eb = c * at1 * n;              // E <- B: +-i k c at1
    const double be = at1 / c * n;              // B <- E: +-i k / c at1
    const double ej = -c * a.mu0 * at1 * n;     // E <- J
    const double bj = a.mu0 * at3 * n;          // B <- J: -+ mu0 i k at3
    // rho / rho_old coefficients: i (..) / |k|^2 * k_b / eps0
    const double k10 = sqrt(a.kzc2[iz] + a.kyc2[iy] + a.kxc2[ix]);
    C2 r10x, r10y, r10z, r11x, r11y, r11z;
    if (m == 0 && k10 == 0.0) {
      const double cdt2 = (c * a.dt) * (c * a.dt);
      const C2 v10{0.0, -1.0 / 3.0 * cdt2 / a.eps0 * n}, v11{0.0, -1.0 / 6.0 * cdt2 / a.eps0 * n};
      r10x = r10y = r10z = v10;
      r11x = r11y = r11z = v11;
    } else {
      const double kk = k10 * k10;
      const double f10 = (at2 - 1.0 / (c * a.dt) * at1) / kk / a.eps0 * n;
      const double f11 = (1.0 / (c * a.dt) * at1 - 1.0) / kk / a.eps0 * n;
      r10x = scl(f10, ik(Kxb)); r10y = scl(f10, ik(Kyb)); r10z = scl(f10, ik(Kzb));
      r11x = scl(f11, ik(Kxb)); r11y = scl(f11, ik(Kyb)); r11z = scl(f11, ik(Kzb));
    }
    C2 v;
    // B from the old E and J
    v = scl(d, bx);
    v = add(v, mul(scl(be, ik(Kzb)), ey));
    v = add(v, mul(scl(-be, ik(Kyb)), ez));
    v = add(v, mul(scl(-bj, ik(Kzb)), jy));
    v = add(v, mul(scl(bj, ik(Kyb)), jz));
    st(a.bx, m, v);
    v = scl(d, by);
    v = add(v, mul(scl(-be, ik(Kzb)), ex));
    v = add(v, mul(scl(be, ik(Kxb)), ez));
    v = add(v, mul(scl(bj, ik(Kzb)), jx));
    v = add(v, mul(scl(-bj, ik(Kxb)), jz));
    st(a.by, m, v);
    v = scl(d, bz);
    v = add(v, mul(scl(be, ik(Kyb)), ex));
    v = add(v, mul(scl(-be, ik(Kxb)), ey));
    v = add(v, mul(scl(-bj, ik(Kyb)), jx));
    v = add(v, mul(scl(bj, ik(Kxb)), jy));
    st(a.bz, m, v);
    // E from the old B, J, rho and rho_old
    v = scl(d, ex);
    v = add(v, mul(scl(-eb, ik(Kzf)), by));
    v = add(v, mul(scl(eb, ik(Kyf)), bz));
    v = add(v, scl(ej, jx));
    v = add(v, mul(r11x, rh));
    v = add(v, mul(r10x, ro));
    st(a.ex, m, v);
    v = scl(d, ey);
    v = add(v, mul(scl(eb, ik(Kzf)), bx));
    v = add(v, mul(scl(-eb, ik(Kxf)), bz));
    v = add(v, scl(ej, jy));
    v = add(v, mul(r11y, rh));
    v = add(v, mul(r10y, ro));
    st(a.ey, m, v);
    v = scl(d, ez);
    v = add(v, mul(scl(-eb, ik(Kyf)), bx));
    v = add(v, mul(scl(eb, ik(Kxf)), by));
    v = add(v, scl(ej, jz));
    v = add(v, mul(r11z, rh));
    v = add(v, mul(r10z, ro));
    st(a.ez, m, v);
  }
}

}  // namespace

extern "C" {

int pxrb_psatd_push(int64_t nkx, int64_t nky, int64_t nkz, double* ex, double* ey, double* ez,
                    double* bx, double* by, double* bz, const double* jx, const double* jy,
                    const double* jz, const double* rho, const double* rhoold,
                    const double* kxf, const double* kxb, const double* kyf, const double* kyb,
                    const double* kzf, const double* kzb, const double* kxc2,
                    const double* kyc2, const double* kzc2, const double* at1,
                    const double* at2, const double* at3, double clight, double eps0,
                    double mu0, double dt, double norm, void* stream) {
  if (nkx < 1 || nky < 1 || nkz < 1) return PXRB_EINVAL;
  const double* in[] = {jx, jy, jz, rho, rhoold, kxf, kxb, kyf, kyb, kzf, kzb,
                        kxc2, kyc2, kzc2, at1, at2, at3};
  for (const double* p : in)
    if (!p) return PXRB_EINVAL;
  if (!ex || !ey || !ez || !bx || !by || !bz) return PXRB_EINVAL;
  if (!(clight > 0.0) || !(dt > 0.0) || !(eps0 > 0.0)) return PXRB_EINVAL;
  PsatdArgs a{nkx, nky, nkz, ex, ey, ez, bx, by, bz, jx, jy, jz, rho, rhoold,
              kxf, kxb, kyf, kyb, kzf, kzb, kxc2, kyc2, kzc2, at1, at2, at3,
              clight, eps0, mu0, dt, norm};
  const i64 nm = nkx * nky * nkz;
  i64 blocks = (nm + 255) / 256;
  if (blocks > 148 * 32) blocks = 148 * 32;
  k_psatd_push<<<(int)blocks, 256, 0, (cudaStream_t)stream>>>(a);
  PXRB_CHECK_LAUNCH();
  return PXRB_OK;
}

}  // extern "C"
