// Hex8 element stiffness for the library (set-up only; the matrix is passed to the kernels by value).
// Follows Hex8Element.CreateKe (src/Mycel.Core/Fem/Hex8Element.cs:98-178): 2x2x2 Gauss points at +-1/sqrt(3),
// weight det(J) = 1/8 for h = 1, Ke(h) = h Ke(1); nu = 0.3 takes the fast path BaseKe * h (:104-112), where
// BaseKe itself is the Gauss-integrated Ke(1, 0.3). Compiled with -ffp-contract=off.
#include <cmath>
#include <cstring>

#include "internal.h"

namespace mycel {
namespace {

void constitutive_unit(double nu, double d[36]) {
  double factor = 1.0 / ((1.0 + nu) * (1.0 - 2.0 * nu));
  double c1 = factor * (1.0 - nu), c2 = factor * nu, c3 = 1.0 / (2.0 * (1.0 + nu));
  for (int i = 0; i < 36; ++i) d[i] = 0.0;
  d[0] = c1; d[1] = c2; d[2] = c2;
  d[6] = c2; d[7] = c1; d[8] = c2;
  d[12] = c2; d[13] = c2; d[14] = c1;
  d[21] = c3; d[28] = c3; d[35] = c3;
}

// strain-displacement matrix (6 x 24) at (xi, eta, zeta) for unit edge, Voigt order xx yy zz yz zx xy
void strain_matrix(double xi, double eta, double zeta, double b[144]) {
  static const double sx[8] = {-1, 1, 1, -1, -1, 1, 1, -1};
  static const double sy[8] = {-1, -1, 1, 1, -1, -1, 1, 1};
  static const double sz[8] = {-1, -1, -1, -1, 1, 1, 1, 1};
  for (int i = 0; i < 144; ++i) b[i] = 0.0;
  const double q = 0.25 * (1.0 / 1.0);
  for (int a = 0; a < 8; ++a) {
    double gx = q * sx[a] * (1.0 + sy[a] * eta) * (1.0 + sz[a] * zeta);
    double gy = q * sy[a] * (1.0 + sx[a] * xi) * (1.0 + sz[a] * zeta);
    double gz = q * sz[a] * (1.0 + sx[a] * xi) * (1.0 + sy[a] * eta);
    b[0 * 24 + 3 * a] = gx;
    b[1 * 24 + 3 * a + 1] = gy;
    b[2 * 24 + 3 * a + 2] = gz;
    b[3 * 24 + 3 * a + 1] = gz;
    b[3 * 24 + 3 * a + 2] = gy;
    b[4 * 24 + 3 * a] = gz;
    b[4 * 24 + 3 * a + 2] = gx;
    b[5 * 24 + 3 * a] = gy;
    b[5 * 24 + 3 * a + 1] = gx;
  }
}

void gauss_ke_unit(double nu, double ke[576]) {
  const double gp = 1.0 / std::sqrt(3.0);
  const double pts[2] = {-gp, gp};
  double d[36], b[144], db[144];
  constitutive_unit(nu, d);
  for (int i = 0; i < 576; ++i) ke[i] = 0.0;
  for (int ix = 0; ix < 2; ++ix)
    for (int iy = 0; iy < 2; ++iy)
      for (int iz = 0; iz < 2; ++iz) {
        strain_matrix(pts[ix], pts[iy], pts[iz], b);
        for (int r = 0; r < 6; ++r)
          for (int c = 0; c < 24; ++c) {
            double s = 0.0;
            for (int k = 0; k < 6; ++k) s += d[r * 6 + k] * b[k * 24 + c];
            db[r * 24 + c] = s;
          }
        for (int i = 0; i < 24; ++i)
          for (int j = 0; j < 24; ++j) {
            double s = 0.0;
            for (int k = 0; k < 6; ++k) s += b[k * 24 + i] * db[k * 24 + j];
            ke[i * 24 + j] += s * (1.0 / 8.0);
          }
      }
}

}  // namespace

void build_ke(double h, double nu, double* ke) {
  if (std::fabs(nu - 0.3) < 1e-15) {
    static double base[576];
    static bool have = false;
    if (!have) {
      gauss_ke_unit(0.3, base);
      have = true;
    }
    for (int i = 0; i < 576; ++i) ke[i] = base[i] * h;
    return;
  }
  gauss_ke_unit(nu, ke);
  if (std::fabs(h - 1.0) > 1e-15)
    for (int i = 0; i < 576; ++i) ke[i] *= h;
}

int64_t num_blocks8192(int64_t n) { return (n + 8191) / 8192; }

// Round an FP32 value to TF32 (10 explicit mantissa bits), to nearest with ties away from zero, as the
// device's cvt.rna.tf32.f32 does; non-finite values pass through.
static float tf32_rna(float v) {
  uint32_t u;
  std::memcpy(&u, &v, 4);
  if ((u & 0x7f800000u) == 0x7f800000u) return v;
  u += 0x1000u;      // half of the 13 dropped bits: ties round away from zero in magnitude
  u &= 0xffffe000u;
  float r;
  std::memcpy(&r, &u, 4);
  return r;
}

void split_ke_tf32(const double* ke, KeTf* out) {
  for (int i = 0; i < 32 * 24; ++i) out->hi[i] = out->lo[i] = 0.0f;
  for (int r = 0; r < 24; ++r)
    for (int c = 0; c < 24; ++c) {
      float f = (float)ke[r * 24 + c];
      float hi = tf32_rna(f);
      out->hi[r * 24 + c] = hi;
      out->lo[r * 24 + c] = tf32_rna(f - hi);
    }
}

// Factorised KE for the FP32 fast path. With trilinear shape functions N_a = phi(x) phi(y) phi(z) on a cube
// and exact (2x2x2 Gauss) integration, every 3x3 block of KE(1, nu) is a sum of Kronecker products of the 1-D
// 2x2 matrices S = int phi'_a phi'_b, M = int phi_a phi_b and C = int phi'_a phi_b:
//   K[i][i] = (lambda + 2 mu) S_i M_j M_k + mu (M_i S_j M_k + M_i M_j S_k)
//   K[i][j] = lambda C_i C^T_j M_k + mu C^T_i C_j M_k                      (i != j, k the third axis)
// (lambda = nu / ((1 + nu)(1 - 2 nu)), mu = 1 / (2 (1 + nu)) for E = 1, as in the constitutive matrix of
// Hex8Element.CreateConstitutiveMatrix, src/Mycel.Core/Fem/Hex8Element.cs:183-215). In the basis
// e = (1, 1), o = (-1, 1) of each axis: S e = 0, S o = 2 o; M e = e / 2, M o = o / 6; C e = o, C o = 0;
// C^T o = e, C^T e = 0. So K is diagonal per component (eigenvalues below) plus one coupling per pair of
// components between basis functions whose parities on the two axes are swapped. Coefficients of an
// element vector in that basis are its 8-point Walsh-Hadamard transform / 8; the h / 8 is folded in here.
void build_hexop64(double h, double nu, HexOpD* out) {
  const double lam = nu / ((1.0 + nu) * (1.0 - 2.0 * nu)), mu = 1.0 / (2.0 * (1.0 + nu));
  const double l2m = lam + 2.0 * mu, sc = h / 8.0;
  const double dcl[2][3] = {{0.0, mu / 2.0, mu / 3.0},
                            {l2m / 2.0, l2m / 6.0 + mu / 6.0, l2m / 18.0 + mu / 9.0}};
  for (int a = 0; a < 2; ++a)
    for (int n = 0; n < 3; ++n) out->dcl[a][n] = dcl[a][n] * sc;
  out->lam[0] = lam / 2.0 * sc;
  out->lam[1] = lam / 6.0 * sc;
  out->mu[0] = mu / 2.0 * sc;
  out->mu[1] = mu / 6.0 * sc;
}

void build_hexop(double h, double nu, HexOpF* out) {
  HexOpD d;
  build_hexop64(h, nu, &d);
  for (int a = 0; a < 2; ++a) {
    for (int n = 0; n < 3; ++n) out->dcl[a][n] = (float)d.dcl[a][n];
    out->lam[a] = (float)d.lam[a];
    out->mu[a] = (float)d.mu[a];
  }
}

}  // namespace mycel
