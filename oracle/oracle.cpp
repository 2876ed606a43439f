// ORACLE — test infrastructure only (see oracle.h). CPU restatement of Mycel.Core's FEM + SIMP inner loop.
// Compiled with -ffp-contract=off -fno-fast-math so every a*b+c rounds twice, as RyuJIT does.
// OpenMP only splits work whose result does not depend on the split (elements of one colour, 8192-blocks,
// filter rows, element-local sensitivities), so any thread count gives the single-thread bits.
#include "oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <unordered_set>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

int g_lane_mode = 0;

void set_msg(char* msg, int len, const char* s) {
  if (msg && len > 0) {
    std::snprintf(msg, (size_t)len, "%s", s);
  }
}

// Vector256<double>.Sum(acc) — lane combine order (runtime switch, see oracle.h).
inline double lane_sum(const double a[4]) {
  switch (g_lane_mode) {
    case 1: return (a[0] + a[2]) + (a[1] + a[3]);
    case 2: return ((a[0] + a[1]) + a[2]) + a[3];
    default: return (a[0] + a[1]) + (a[2] + a[3]);
  }
}

// Math.Pow as used on the path (E_e = Emin + rho^p (E0-Emin), dE/drho = p rho^(p-1) dE): .NET on Linux calls
// the C runtime's pow. Called through a volatile pointer so the compiler cannot replace a call whose exponent
// it can see (pow(x, 2.0) -> x * x) by its own arithmetic.
double (*volatile g_libm_pow)(double, double) = ::pow;
double mpow(double x, double y) { return g_libm_pow(x, y); }

}  // namespace

// ---------------------------------------------------------------------------------------------------------
// Hex8Element — src/Mycel.Core/Fem/Hex8Element.cs:50-215
// ---------------------------------------------------------------------------------------------------------
namespace {
const double kXi[8] = {-1, 1, 1, -1, -1, 1, 1, -1};
const double kEta[8] = {-1, -1, 1, 1, -1, -1, 1, 1};
const double kZeta[8] = {-1, -1, -1, -1, 1, 1, 1, 1};

// Hex8Element.CreateConstitutiveMatrix (Hex8Element.cs:77-92)
void constitutive(double e, double nu, double d[36]) {
  double factor = e / ((1.0 + nu) * (1.0 - 2.0 * nu));
  double c1 = factor * (1.0 - nu);
  double c2 = factor * nu;
  double c3 = e / (2.0 * (1.0 + nu));
  for (int i = 0; i < 36; ++i) d[i] = 0.0;
  d[0] = c1; d[1] = c2; d[2] = c2;
  d[6] = c2; d[7] = c1; d[8] = c2;
  d[12] = c2; d[13] = c2; d[14] = c1;
  d[21] = c3; d[28] = c3; d[35] = c3;
}

// Hex8Element.EvaluateB (Hex8Element.cs:183-215)
void evaluate_b(double xi, double eta, double zeta, double h, double b[144]) {
  for (int i = 0; i < 144; ++i) b[i] = 0.0;
  double invH = 1.0 / h;
  for (int a = 0; a < 8; ++a) {
    double dNdx = (0.25 * invH) * kXi[a] * (1.0 + kEta[a] * eta) * (1.0 + kZeta[a] * zeta);
    double dNdy = (0.25 * invH) * kEta[a] * (1.0 + kXi[a] * xi) * (1.0 + kZeta[a] * zeta);
    double dNdz = (0.25 * invH) * kZeta[a] * (1.0 + kXi[a] * xi) * (1.0 + kEta[a] * eta);
    int cu = 3 * a, cv = 3 * a + 1, cw = 3 * a + 2;
    b[0 * 24 + cu] = dNdx;
    b[1 * 24 + cv] = dNdy;
    b[2 * 24 + cw] = dNdz;
    b[3 * 24 + cv] = dNdz;
    b[3 * 24 + cw] = dNdy;
    b[4 * 24 + cu] = dNdz;
    b[4 * 24 + cw] = dNdx;
    b[5 * 24 + cu] = dNdy;
    b[5 * 24 + cv] = dNdx;
  }
}

// Gauss-integrated Ke(1, nu) (Hex8Element.cs:114-166), scaled by h when |h-1| > 1e-15 (:169-175).
void create_ke_gauss(double h, double nu, double ke[576]) {
  const double g[2] = {-1.0 / std::sqrt(3.0), 1.0 / std::sqrt(3.0)};
  double d[36], b[144], db[144];
  constitutive(1.0, nu, d);
  for (int i = 0; i < 576; ++i) ke[i] = 0.0;
  const double dV = 1.0 / 8.0;
  for (int ix = 0; ix < 2; ++ix)
    for (int iy = 0; iy < 2; ++iy)
      for (int iz = 0; iz < 2; ++iz) {
        evaluate_b(g[ix], g[iy], g[iz], 1.0, b);
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
            ke[i * 24 + j] += s * dV;
          }
      }
  if (std::fabs(h - 1.0) > 1e-15)
    for (int i = 0; i < 576; ++i) ke[i] *= h;
}

const double* base_ke() {
  static double ke[576];
  static bool init = false;
  if (!init) {
    create_ke_gauss(1.0, 0.3, ke);  // BaseKe is built before the nu=0.3 fast path exists (Hex8Element.cs:60)
    init = true;
  }
  return ke;
}
}  // namespace

extern "C" int orc_create_ke(double h, double nu, double* ke) {
  if (!(h > 0)) return ORC_E_ARG;
  if (std::fabs(nu - 0.3) < 1e-15) {  // fast path (Hex8Element.cs:104-112)
    const double* bk = base_ke();
    for (int i = 0; i < 576; ++i) ke[i] = bk[i] * h;
    return ORC_OK;
  }
  create_ke_gauss(h, nu, ke);
  return ORC_OK;
}

// ---------------------------------------------------------------------------------------------------------
// FeModel — src/Mycel.Core/Fem/FeModel.cs:43-184, AssembleForces :263-321
// ---------------------------------------------------------------------------------------------------------
struct orc_load {
  std::vector<int32_t> nodes;
  std::vector<double> areas;
  float f[3];
};

struct orc_model {
  int nx, ny, nz;
  float h;
  std::vector<uint8_t> domain;
  double e0, nu, emin_ratio, emin;
  std::vector<int32_t> fixed;
  std::vector<orc_load> loads;
  std::vector<double> density;
  double penal;
  int64_t total_elements, total_nodes, total_dofs;
  std::vector<int32_t> active_elements;
  std::vector<int32_t> by_color[8];
  std::vector<uint8_t> active_nodes;
  std::vector<uint8_t> constrained;
  int64_t active_node_count = 0, active_fixed_count = 0;
};

extern "C" orc_model* orc_model_create(int nx, int ny, int nz, float h, const uint8_t* domain, double e0, double nu,
                                       double emin_ratio, const int32_t* fixed, int32_t n_fixed,
                                       const double* element_density, double penal, int* status, char* msg,
                                       int msglen) {
  *status = ORC_OK;
  if (nx <= 0 || ny <= 0 || nz <= 0 || !(h > 0.0f)) {
    *status = ORC_E_ARG;
    set_msg(msg, msglen, "Grid dimensions must be strictly positive.");
    return nullptr;
  }
  orc_model* m = new orc_model();
  m->nx = nx; m->ny = ny; m->nz = nz; m->h = h;
  m->total_elements = (int64_t)nx * ny * nz;
  m->total_nodes = (int64_t)(nx + 1) * (ny + 1) * (nz + 1);
  m->total_dofs = 3 * m->total_nodes;
  m->domain.assign(domain, domain + m->total_elements);
  m->e0 = e0; m->nu = nu; m->emin_ratio = emin_ratio; m->emin = e0 * emin_ratio;  // FeMaterial.cs:16
  m->penal = penal;
  if (element_density) m->density.assign(element_density, element_density + m->total_elements);
  else m->density.assign(m->total_elements, 1.0);
  m->active_nodes.assign(m->total_nodes, 0);
  int nx1 = nx + 1, ny1 = ny + 1;
  for (int iz = 0; iz < nz; ++iz) {
    int cz = (iz & 1) << 2;
    for (int iy = 0; iy < ny; ++iy) {
      int cyz = cz | ((iy & 1) << 1);
      for (int ix = 0; ix < nx; ++ix) {
        int e = ix + nx * (iy + ny * iz);
        if (m->domain[e] != 0) {
          m->active_elements.push_back(e);
          m->by_color[cyz | (ix & 1)].push_back(e);
          int n0 = ix + nx1 * (iy + ny1 * iz);
          int n4 = n0 + nx1 * ny1;
          int ns[8] = {n0, n0 + 1, n0 + nx1 + 1, n0 + nx1, n4, n4 + 1, n4 + nx1 + 1, n4 + nx1};
          for (int a = 0; a < 8; ++a) m->active_nodes[ns[a]] = 1;
        }
      }
    }
  }
  for (int64_t n = 0; n < m->total_nodes; ++n) m->active_node_count += m->active_nodes[n];
  m->constrained.assign(m->total_dofs, 0);
  for (int64_t n = 0; n < m->total_nodes; ++n)
    if (!m->active_nodes[n]) m->constrained[3 * n] = m->constrained[3 * n + 1] = m->constrained[3 * n + 2] = 1;
  std::unordered_set<int32_t> act_fixed;
  for (int32_t i = 0; i < n_fixed; ++i) {
    int32_t dof = fixed[i];
    if ((uint64_t)(uint32_t)dof < (uint64_t)m->total_dofs && dof >= 0) {
      m->constrained[dof] = 1;
      if (m->active_nodes[dof / 3]) act_fixed.insert(dof);
    } else {
      char buf[160];
      std::snprintf(buf, sizeof buf, "Fixed DOF %d is out of bounds [0, %lld].", dof, (long long)(m->total_dofs - 1));
      set_msg(msg, msglen, buf);
      *status = ORC_E_ARG;
      delete m;
      return nullptr;
    }
    m->fixed.push_back(dof);
  }
  m->active_fixed_count = (int64_t)act_fixed.size();
  return m;
}

extern "C" int orc_model_add_load(orc_model* m, int32_t n_nodes, const int32_t* nodes, const double* areas, float fx,
                                  float fy, float fz) {
  orc_load l;
  l.nodes.assign(nodes, nodes + n_nodes);
  l.areas.assign(areas, areas + n_nodes);
  l.f[0] = fx; l.f[1] = fy; l.f[2] = fz;
  m->loads.push_back(l);
  return ORC_OK;
}

extern "C" void orc_model_free(orc_model* m) { delete m; }

extern "C" void orc_model_counts(const orc_model* m, int64_t* o) {
  o[0] = (int64_t)m->active_elements.size();
  o[1] = m->active_node_count;
  o[2] = m->active_fixed_count;
  o[3] = m->total_dofs;
  o[4] = m->total_elements;
  o[5] = m->total_nodes;
}

extern "C" void orc_model_active_elements(const orc_model* m, int32_t* out) {
  std::copy(m->active_elements.begin(), m->active_elements.end(), out);
}

extern "C" void orc_model_constrained(const orc_model* m, uint8_t* out) {
  std::copy(m->constrained.begin(), m->constrained.end(), out);
}

extern "C" void orc_model_set_density(orc_model* m, const double* d, double penal) {
  std::copy(d, d + m->total_elements, m->density.begin());
  m->penal = penal;
}

// One load case's nodal forces added into f (the body of FeModel.AssembleForces' loop, FeModel.cs:267-318)
static int add_load_case(const orc_model* m, const orc_load& l, double* f, char* msg, int msglen) {
  int n = (int)l.nodes.size();
  if (n == 0) {
    if (l.f[0] != 0.0f || l.f[1] != 0.0f || l.f[2] != 0.0f) {
      set_msg(msg, msglen, "Cannot assemble load case: surface patch contains 0 nodes.");
      return ORC_E_INVALID_OPERATION;
    }
    return ORC_OK;
  }
  double total = 0.0;
  for (int i = 0; i < n; ++i) total += l.areas[i];
  for (int i = 0; i < n; ++i)
    if ((uint64_t)(uint32_t)l.nodes[i] >= (uint64_t)m->total_nodes || l.nodes[i] < 0) {
      set_msg(msg, msglen, "Patch node index is out of bounds.");
      return ORC_E_INVALID_OPERATION;
    }
  if (total <= 0.0) {
    double inv = 1.0 / n;
    double fx = (double)l.f[0] * inv, fy = (double)l.f[1] * inv, fz = (double)l.f[2] * inv;
    for (int i = 0; i < n; ++i) {
      int64_t nd = l.nodes[i];
      f[3 * nd] += fx; f[3 * nd + 1] += fy; f[3 * nd + 2] += fz;
    }
  } else {
    double inv = 1.0 / total;
    for (int i = 0; i < n; ++i) {
      int64_t nd = l.nodes[i];
      double w = l.areas[i] * inv;
      f[3 * nd] += (double)l.f[0] * w;
      f[3 * nd + 1] += (double)l.f[1] * w;
      f[3 * nd + 2] += (double)l.f[2] * w;
    }
  }
  return ORC_OK;
}

// FeModel.AssembleForces (FeModel.cs:263-321): all load cases summed into one vector, in case order
extern "C" int orc_model_assemble_forces(const orc_model* m, double* f, char* msg, int msglen) {
  for (int64_t i = 0; i < m->total_dofs; ++i) f[i] = 0.0;
  for (const orc_load& l : m->loads) {
    int st = add_load_case(m, l, f, msg, msglen);
    if (st) return st;
  }
  return ORC_OK;
}

// Load case k alone (the same arithmetic on a zero vector): the right-hand side of case k when load cases are
// kept separate (no counterpart in the reference, which sums them)
extern "C" int orc_model_assemble_case_forces(const orc_model* m, int32_t k, double* f, char* msg, int msglen) {
  if (k < 0 || k >= (int32_t)m->loads.size()) {
    set_msg(msg, msglen, "Load case index is out of range.");
    return ORC_E_ARG;
  }
  for (int64_t i = 0; i < m->total_dofs; ++i) f[i] = 0.0;
  return add_load_case(m, m->loads[k], f, msg, msglen);
}

extern "C" int32_t orc_model_load_case_count(const orc_model* m) { return (int32_t)m->loads.size(); }

// ---------------------------------------------------------------------------------------------------------
// FemOperator — src/Mycel.Core/Fem/FemOperator.cs:33-294, 379-439
// ---------------------------------------------------------------------------------------------------------
struct orc_op {
  orc_model* m;
  double ke[576];
  double diag_ke[24];
  std::vector<double> diag_a;
  std::vector<int32_t> dofs[8];
  std::vector<double> ev[8];
};

namespace {
void element_dofs(const orc_model* m, int e, int32_t* dofs) {
  int nx = m->nx, ny = m->ny, nx1 = nx + 1, ny1 = ny + 1;
  int nxny = nx * ny;
  int iz = e / nxny, rem = e % nxny, iy = rem / nx, ix = rem % nx;  // GridSpec.InverseElementIndex
  int n0 = ix + nx1 * (iy + ny1 * iz);
  int n4 = n0 + nx1 * ny1;
  int ns[8] = {n0, n0 + 1, n0 + nx1 + 1, n0 + nx1, n4, n4 + 1, n4 + nx1 + 1, n4 + nx1};
  for (int a = 0; a < 8; ++a) {
    dofs[3 * a] = 3 * ns[a];
    dofs[3 * a + 1] = 3 * ns[a] + 1;
    dofs[3 * a + 2] = 3 * ns[a] + 2;
  }
}

// FemOperator.AssembleDiagonal (FemOperator.cs:143-172)
void assemble_diagonal(orc_op* op) {
  std::fill(op->diag_a.begin(), op->diag_a.end(), 0.0);
  for (int c = 0; c < 8; ++c) {
    size_t cnt = op->m->by_color[c].size();
    for (size_t i = 0; i < cnt; ++i) {
      double ee = op->ev[c][i];
      for (int k = 0; k < 24; ++k) op->diag_a[op->dofs[c][i * 24 + k]] += ee * op->diag_ke[k];
    }
  }
  for (int64_t i = 0; i < op->m->total_dofs; ++i)
    if (op->m->constrained[i]) op->diag_a[i] = 1.0;
}

// FemOperator.MultiplyElementUnsafe, AVX2 branch (FemOperator.cs:379-422): ue = x*E, then per row four lane
// accumulators acc_l = ((((k0*u0 + k1*u1) + k2*u2) + k3*u3) + k4*u4) + k5*u5 over columns l, l+4, ..., l+20,
// combined by Vector256.Sum and added to y.
inline void multiply_element(const double* ke, const int32_t* dofs, double ee, const double* x, double* y) {
  double ue[24];
  for (int k = 0; k < 24; ++k) ue[k] = x[dofs[k]] * ee;
  for (int r = 0; r < 24; ++r) {
    const double* row = ke + r * 24;
    double acc[4];
    for (int l = 0; l < 4; ++l) {
      double s = row[l] * ue[l] + row[4 + l] * ue[4 + l];
      s = s + row[8 + l] * ue[8 + l];
      s = s + row[12 + l] * ue[12 + l];
      s = s + row[16 + l] * ue[16 + l];
      s = s + row[20 + l] * ue[20 + l];
      acc[l] = s;
    }
    y[dofs[r]] += lane_sum(acc);
  }
}
}  // namespace

extern "C" orc_op* orc_op_create(orc_model* m) {
  orc_op* op = new orc_op();
  op->m = m;
  orc_create_ke((double)m->h, m->nu, op->ke);
  for (int i = 0; i < 24; ++i) op->diag_ke[i] = op->ke[i * 24 + i];
  op->diag_a.assign(m->total_dofs, 0.0);
  for (int c = 0; c < 8; ++c) {
    size_t cnt = m->by_color[c].size();
    op->dofs[c].resize(cnt * 24);
    op->ev[c].resize(cnt);
    for (size_t i = 0; i < cnt; ++i) {
      int e = m->by_color[c][i];
      element_dofs(m, e, &op->dofs[c][i * 24]);
      op->ev[c][i] = m->emin + mpow(m->density[e], m->penal) * (m->e0 - m->emin);  // FemOperator.cs:100
    }
  }
  assemble_diagonal(op);
  return op;
}

extern "C" void orc_op_free(orc_op* op) { delete op; }

// FemOperator.UpdateDensities (FemOperator.cs:114-138)
extern "C" void orc_op_update_densities(orc_op* op, const double* d, double penal) {
  orc_model* m = op->m;
  if (d != m->density.data()) std::copy(d, d + m->total_elements, m->density.begin());
  m->penal = penal;
  for (int c = 0; c < 8; ++c) {
    size_t cnt = m->by_color[c].size();
    for (size_t i = 0; i < cnt; ++i) op->ev[c][i] = m->emin + mpow(d[m->by_color[c][i]], penal) * (m->e0 - m->emin);
  }
  assemble_diagonal(op);
}

extern "C" void orc_op_diag(const orc_op* op, double* out) { std::copy(op->diag_a.begin(), op->diag_a.end(), out); }

extern "C" void orc_op_element_e(const orc_op* op, double* e_box) {
  for (int64_t e = 0; e < op->m->total_elements; ++e) e_box[e] = 0.0;
  for (int c = 0; c < 8; ++c)
    for (size_t i = 0; i < op->m->by_color[c].size(); ++i) e_box[op->m->by_color[c][i]] = op->ev[c][i];
}

// FemOperator.ApplyK (FemOperator.cs:196-243): colours in order; elements of one colour share no node.
extern "C" void orc_op_apply_k(orc_op* op, const double* x, double* y) {
  int64_t n = op->m->total_dofs;
  for (int64_t i = 0; i < n; ++i) y[i] = 0.0;
  for (int c = 0; c < 8; ++c) {
    int64_t cnt = (int64_t)op->m->by_color[c].size();
    const int32_t* dofs = op->dofs[c].data();
    const double* ev = op->ev[c].data();
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < cnt; ++i) multiply_element(op->ke, dofs + i * 24, ev[i], x, y);
  }
}

// FemOperator.ApplyKScalarReference (FemOperator.cs:299-366): dot then scale, sequential columns.
extern "C" void orc_op_apply_k_scalar_reference(orc_op* op, const double* x, double* y) {
  orc_model* m = op->m;
  for (int64_t i = 0; i < m->total_dofs; ++i) y[i] = 0.0;
  int32_t dofs[24];
  double ue[24], ye[24];
  for (int e : m->active_elements) {
    element_dofs(m, e, dofs);
    double ee = m->emin + mpow(m->density[e], m->penal) * (m->e0 - m->emin);
    for (int k = 0; k < 24; ++k) ue[k] = x[dofs[k]];
    for (int r = 0; r < 24; ++r) {
      double s = 0.0;
      for (int c = 0; c < 24; ++c) s += op->ke[r * 24 + c] * ue[c];
      ye[r] = s * ee;
    }
    for (int k = 0; k < 24; ++k) y[dofs[k]] += ye[k];
  }
}

// FemOperator.ApplyA (FemOperator.cs:250-294)
extern "C" void orc_op_apply_a(orc_op* op, const double* x, double* y, int projected) {
  orc_model* m = op->m;
  int64_t n = m->total_dofs;
  if (projected) {
    orc_op_apply_k(op, x, y);
    for (int32_t dof : m->fixed) y[dof] = x[dof];
  } else {
    std::vector<double> v(n);
    for (int64_t i = 0; i < n; ++i) v[i] = m->constrained[i] ? 0.0 : x[i];
    orc_op_apply_k(op, v.data(), y);
    for (int64_t i = 0; i < n; ++i)
      if (m->constrained[i]) y[i] = x[i];
  }
}

// ---------------------------------------------------------------------------------------------------------
// PcgSolver — src/Mycel.Core/Fem/PcgSolver.cs:80-553 (Jacobi preconditioner JacobiPreconditioner.cs:15-27)
// ---------------------------------------------------------------------------------------------------------
namespace {
const int kBlock = 8192;  // PcgSolver.cs:18

// Chunk bodies (PcgSolver.cs:424-553): four lane accumulators over the 4-aligned part, Vector256.Sum,
// then the scalar tail. Partial sums are added block by block (ReducePartialSums :414-422).
double dot_blocks(const double* a, const double* b, int64_t n, std::vector<double>& part) {
  int64_t nb = (n + kBlock - 1) / kBlock;
  part.assign(nb, 0.0);
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < nb; ++k) {
    int64_t s0 = k * kBlock, cnt = std::min<int64_t>(kBlock, n - s0);
    const double *pa = a + s0, *pb = b + s0;
    int64_t vc = cnt / 4;
    double acc[4] = {0, 0, 0, 0};
    for (int64_t i = 0; i < vc; ++i)
      for (int l = 0; l < 4; ++l) acc[l] = acc[l] + pa[4 * i + l] * pb[4 * i + l];
    double s = lane_sum(acc);
    for (int64_t i = vc * 4; i < cnt; ++i) s += pa[i] * pb[i];
    part[k] = s;
  }
  double sum = 0.0;
  for (int64_t k = 0; k < nb; ++k) sum += part[k];
  return sum;
}

double update_xr_norm(double* x, double* r, const double* p, const double* ap, double alpha, int64_t n,
                      std::vector<double>& part) {
  int64_t nb = (n + kBlock - 1) / kBlock;
  part.assign(nb, 0.0);
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < nb; ++k) {
    int64_t s0 = k * kBlock, cnt = std::min<int64_t>(kBlock, n - s0);
    double *px = x + s0, *pr = r + s0;
    const double *pp = p + s0, *pap = ap + s0;
    int64_t vc = cnt / 4;
    double acc[4] = {0, 0, 0, 0};
    for (int64_t i = 0; i < vc; ++i)
      for (int l = 0; l < 4; ++l) {
        int64_t j = 4 * i + l;
        double vx = px[j] + alpha * pp[j];
        double vr = pr[j] - alpha * pap[j];
        px[j] = vx;
        pr[j] = vr;
        acc[l] = acc[l] + vr * vr;
      }
    double s = lane_sum(acc);
    for (int64_t j = vc * 4; j < cnt; ++j) {
      double xi = px[j] + alpha * pp[j];
      double ri = pr[j] - alpha * pap[j];
      px[j] = xi;
      pr[j] = ri;
      s += ri * ri;
    }
    part[k] = s;
  }
  double sum = 0.0;
  for (int64_t k = 0; k < nb; ++k) sum += part[k];
  return sum;
}

double apply_prec_dot(const double* r, double* z, const double* inv, int64_t n, std::vector<double>& part) {
  int64_t nb = (n + kBlock - 1) / kBlock;
  part.assign(nb, 0.0);
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < nb; ++k) {
    int64_t s0 = k * kBlock, cnt = std::min<int64_t>(kBlock, n - s0);
    const double *pr = r + s0, *pi = inv + s0;
    double* pz = z + s0;
    int64_t vc = cnt / 4;
    double acc[4] = {0, 0, 0, 0};
    for (int64_t i = 0; i < vc; ++i)
      for (int l = 0; l < 4; ++l) {
        int64_t j = 4 * i + l;
        double vz = pr[j] * pi[j];
        pz[j] = vz;
        acc[l] = acc[l] + pr[j] * vz;
      }
    double s = lane_sum(acc);
    for (int64_t j = vc * 4; j < cnt; ++j) {
      double zi = pr[j] * pi[j];
      pz[j] = zi;
      s += pr[j] * zi;
    }
    part[k] = s;
  }
  double sum = 0.0;
  for (int64_t k = 0; k < nb; ++k) sum += part[k];
  return sum;
}

void fmt_e3(char* out, size_t len, const char* pre, double v, const char* post) {
  // .NET "E3" format: d.dddE+ddd
  char buf[64];
  std::snprintf(buf, sizeof buf, "%.3E", v);
  // C prints E+dd; .NET prints E+ddd
  char* e = std::strchr(buf, 'E');
  if (e && std::isfinite(v)) {
    char sign = e[1];
    int ex = std::atoi(e + 2);
    std::snprintf(e, sizeof buf - (size_t)(e - buf), "E%c%03d", sign, ex);
  }
  std::snprintf(out, len, "%s%s%s", pre, buf, post);
}
}  // namespace

extern "C" int orc_pcg_solve(orc_op* op, const double* b, double* x, double tol, int32_t max_iter,
                             orc_pcg_result* res, char* msg, int msglen) {
  orc_model* m = op->m;
  std::memset(res, 0, sizeof *res);
  if (m->active_fixed_count < 6) {  // PcgSolver.cs:95-100
    char buf[256];
    std::snprintf(buf, sizeof buf,
                  "Model has fewer than 6 unique fixed DOFs on active nodes (found %lld). At least 6 fixed DOFs are "
                  "required to prevent rigid body modes in 3D.",
                  (long long)m->active_fixed_count);
    set_msg(msg, msglen, buf);
    return ORC_E_UNDERCONSTRAINED;
  }
  int64_t n = m->total_dofs;
  const uint8_t* con = m->constrained.data();
  bool nonzero = false;
  for (int64_t i = 0; i < n; ++i) {
    if (con[i]) x[i] = 0.0;
    else if (x[i] != 0.0) nonzero = true;
  }
  double bn2 = 0.0;
  for (int64_t i = 0; i < n; ++i)
    if (!con[i]) bn2 += b[i] * b[i];
  double bnorm = std::sqrt(bn2);
  if (bnorm <= 1e-30) {
    for (int64_t i = 0; i < n; ++i) x[i] = 0.0;
    res->converged = 1;
    std::snprintf(res->message, sizeof res->message, "RHS is zero. Solution is zero.");
    return ORC_OK;
  }
  std::vector<double> inv(n), r(n), z(n), p(n), ap(n), part;
  for (int64_t i = 0; i < n; ++i) {
    double d = op->diag_a[i];
    inv[i] = std::fabs(d) > 1e-30 ? 1.0 / d : 1.0;
  }
  double rn2;
  if (nonzero) {
    orc_op_apply_a(op, x, ap.data(), 1);
    for (int64_t i = 0; i < n; ++i) r[i] = con[i] ? 0.0 : (b[i] - ap[i]);
    rn2 = dot_blocks(r.data(), r.data(), n, part);
  } else {
    for (int64_t i = 0; i < n; ++i) r[i] = con[i] ? 0.0 : b[i];
    rn2 = bn2;
  }
  double rel = std::sqrt(rn2) / bnorm;
  if (rel <= tol) {
    res->final_residual = rel;
    res->converged = 1;
    std::snprintf(res->message, sizeof res->message, "Initial guess already converged.");
    return ORC_OK;
  }
  double rho0 = apply_prec_dot(r.data(), z.data(), inv.data(), n, part);
  p = z;
  int iter = 0;
  double prev = rel;
  int stag = 0;
  while (iter < max_iter) {
    ++iter;
    orc_op_apply_a(op, p.data(), ap.data(), 1);
    double pap = dot_blocks(p.data(), ap.data(), n, part);
    if (!(pap > 1e-30) || !std::isfinite(pap)) {
      res->iterations = iter;
      res->final_residual = rel;
      fmt_e3(res->message, sizeof res->message, "PCG curvature breakdown (p\xe1\xb5\x80" "Ap = ", pap,
             " <= 0). Is the model not sufficiently constrained?");
      return ORC_OK;
    }
    double alpha = rho0 / pap;
    if (!std::isfinite(alpha) || alpha <= 0.0) {
      res->iterations = iter;
      res->final_residual = rel;
      fmt_e3(res->message, sizeof res->message, "PCG step breakdown (alpha = ", alpha,
             "). Is the model not sufficiently constrained?");
      return ORC_OK;
    }
    rn2 = update_xr_norm(x, r.data(), p.data(), ap.data(), alpha, n, part);
    rel = std::sqrt(rn2) / bnorm;
    if (rel <= tol) {
      res->iterations = iter;
      res->final_residual = rel;
      res->converged = 1;
      return ORC_OK;
    }
    if (std::fabs(rel - prev) < 1e-15 * rel) {
      if (++stag > 50) {
        res->iterations = iter;
        res->final_residual = rel;
        std::snprintf(res->message, sizeof res->message,
                      "PCG stagnated: residual stopped decreasing. Is the model not sufficiently constrained?");
        return ORC_OK;
      }
    } else {
      stag = 0;
    }
    prev = rel;
    double rho1 = apply_prec_dot(r.data(), z.data(), inv.data(), n, part);
    double beta = rho1 / rho0;
    if (!std::isfinite(beta) || beta < 0.0) {
      res->iterations = iter;
      res->final_residual = rel;
      fmt_e3(res->message, sizeof res->message, "PCG search direction breakdown (beta = ", beta,
             "). Is the model not sufficiently constrained?");
      return ORC_OK;
    }
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
    rho0 = rho1;
  }
  res->iterations = iter;
  res->final_residual = rel;
  std::snprintf(res->message, sizeof res->message,
                "PCG reached maximum iterations without converging. Is the model not sufficiently constrained?");
  return ORC_OK;
}

// ---------------------------------------------------------------------------------------------------------
// StaticAnalysis.Run — src/Mycel.Core/Fem/StaticAnalysis.cs:35-142
// ---------------------------------------------------------------------------------------------------------
extern "C" int orc_static_run(orc_model* m, double tol, int32_t max_iter, const double* warm, int64_t warm_len,
                              int throw_nc, double* u, double* reactions, double* compliance, double* max_disp,
                              orc_pcg_result* res, char* msg, int msglen) {
  if (m->active_fixed_count < 6) {
    char buf[256];
    std::snprintf(buf, sizeof buf,
                  "Model has fewer than 6 unique fixed DOFs on active nodes (found %lld). At least 6 fixed DOFs are "
                  "required to prevent rigid body modes in 3D.",
                  (long long)m->active_fixed_count);
    set_msg(msg, msglen, buf);
    return ORC_E_UNDERCONSTRAINED;
  }
  int64_t n = m->total_dofs;
  std::vector<double> f(n), b(n);
  int st = orc_model_assemble_forces(m, f.data(), msg, msglen);
  if (st) return st;
  for (int64_t i = 0; i < n; ++i) b[i] = m->constrained[i] ? 0.0 : f[i];
  for (int64_t i = 0; i < n; ++i) u[i] = 0.0;
  if (warm) {
    if (warm_len != n) {
      char buf[200];
      std::snprintf(buf, sizeof buf, "WarmStartDisplacements length (%lld) must match TotalDofs (%lld).",
                    (long long)warm_len, (long long)n);
      set_msg(msg, msglen, buf);
      return ORC_E_ARG;
    }
    std::copy(warm, warm + n, u);
  }
  orc_op* op = orc_op_create(m);
  st = orc_pcg_solve(op, b.data(), u, tol, max_iter, res, msg, msglen);
  if (st) {
    orc_op_free(op);
    return st;
  }
  if (throw_nc && !res->converged) {
    char buf[400];
    std::snprintf(buf, sizeof buf,
                  "FEM solver did not converge in %d iterations (%s). Is the model not sufficiently constrained?",
                  res->iterations, res->message);
    set_msg(msg, msglen, buf);
    orc_op_free(op);
    return ORC_E_NOT_CONVERGED;
  }
  double c = 0.0;
  for (int64_t i = 0; i < n; ++i) c += f[i] * u[i];
  *compliance = c;
  if (reactions) {
    std::vector<double> ku(n);
    orc_op_apply_k(op, u, ku.data());
    for (int64_t i = 0; i < n; ++i) reactions[i] = 0.0;
    for (int32_t d : m->fixed) reactions[d] = ku[d];
  }
  double md = 0.0;
  for (int64_t nd = 0; nd < m->total_nodes; ++nd)
    if (m->active_nodes[nd]) {
      double ux = u[3 * nd], uy = u[3 * nd + 1], uz = u[3 * nd + 2];
      double s = ux * ux + uy * uy + uz * uz;
      if (s > md) md = s;
    }
  *max_disp = std::sqrt(md);
  orc_op_free(op);
  return ORC_OK;
}

// StaticAnalysis.ComputeElementVonMises (StaticAnalysis.cs:144-216)
extern "C" void orc_von_mises(orc_op* op, const double* u, double* vm) {
  orc_model* m = op->m;
  for (int64_t e = 0; e < m->total_elements; ++e) vm[e] = 0.0;
  double invH = 1.0 / (double)m->h;
  double bc[144], d[36];
  evaluate_b(0.0, 0.0, 0.0, 1.0, bc);
  constitutive(1.0, m->nu, d);
  for (int c = 0; c < 8; ++c)
    for (size_t i = 0; i < m->by_color[c].size(); ++i) {
      int e = m->by_color[c][i];
      double ee = op->ev[c][i];
      const int32_t* dofs = &op->dofs[c][i * 24];
      double ue[24], eps[6], sig[6];
      for (int k = 0; k < 24; ++k) ue[k] = u[dofs[k]];
      for (int r = 0; r < 6; ++r) {
        double s = 0.0;
        for (int k = 0; k < 24; ++k) s += bc[r * 24 + k] * ue[k];
        eps[r] = s * invH;
      }
      for (int r = 0; r < 6; ++r) {
        double s = 0.0;
        for (int k = 0; k < 6; ++k) s += d[r * 6 + k] * eps[k];
        sig[r] = s * ee;
      }
      double d1 = sig[0] - sig[1], d2 = sig[1] - sig[2], d3 = sig[2] - sig[0];
      vm[e] = std::sqrt(0.5 * (d1 * d1 + d2 * d2 + d3 * d3) +
                        3.0 * (sig[3] * sig[3] + sig[4] * sig[4] + sig[5] * sig[5]));
    }
}

// ---------------------------------------------------------------------------------------------------------
// DensityFilter — src/Mycel.Core/Optimization/DensityFilter.cs:34-303
// ---------------------------------------------------------------------------------------------------------
struct orc_filter {
  int32_t n;
  std::vector<int32_t> fo, fc, ao, ac;
  std::vector<double> fw, aw, s;
};

extern "C" orc_filter* orc_filter_create(int nx, int ny, int nz, const uint8_t* domain, const int32_t* active,
                                         int32_t n_active, double rmin) {
  orc_filter* f = new orc_filter();
  f->n = n_active;
  int64_t total = (int64_t)nx * ny * nz;
  std::vector<int32_t> e2a(total, -1);
  for (int32_t i = 0; i < n_active; ++i) e2a[active[i]] = i;
  int rc = (int)std::ceil(rmin);
  double rsq = rmin * rmin;
  std::vector<std::vector<int32_t>> rc_cols(n_active);
  std::vector<std::vector<double>> rc_w(n_active);
#pragma omp parallel for schedule(dynamic, 256)
  for (int32_t ei = 0; ei < n_active; ++ei) {
    int e = active[ei];
    int ez = e / (nx * ny), rem = e % (nx * ny), ey = rem / nx, ex = rem % nx;
    double hs = 0.0;
    int x0 = std::max(0, ex - rc), x1 = std::min(nx - 1, ex + rc);
    int y0 = std::max(0, ey - rc), y1 = std::min(ny - 1, ey + rc);
    int z0 = std::max(0, ez - rc), z1 = std::min(nz - 1, ez + rc);
    for (int jz = z0; jz <= z1; ++jz) {
      int dz = jz - ez, dzs = dz * dz;
      for (int jy = y0; jy <= y1; ++jy) {
        int dy = jy - ey, dyzs = dzs + dy * dy;
        for (int jx = x0; jx <= x1; ++jx) {
          int dx = jx - ex, ds = dyzs + dx * dx;
          if ((double)ds < rsq) {
            int nb = jx + nx * (jy + ny * jz);
            if (domain[nb] != 0) {
              int ni = e2a[nb];
              if (ni >= 0) {
                double dist = std::sqrt((double)ds);
                if (dist < rmin) {
                  double w = rmin - dist;
                  rc_cols[ei].push_back(ni);
                  rc_w[ei].push_back(w);
                  hs += w;
                }
              }
            }
          }
        }
      }
    }
    double inv = hs > 0.0 ? 1.0 / hs : 1.0;
    for (double& w : rc_w[ei]) w *= inv;
  }
  f->fo.assign(n_active + 1, 0);
  int64_t nnz = 0;
  for (int32_t i = 0; i < n_active; ++i) {
    f->fo[i] = (int32_t)nnz;
    nnz += (int64_t)rc_cols[i].size();
  }
  f->fo[n_active] = (int32_t)nnz;
  f->fc.resize(nnz);
  f->fw.resize(nnz);
  for (int32_t i = 0; i < n_active; ++i) {
    std::copy(rc_cols[i].begin(), rc_cols[i].end(), f->fc.begin() + f->fo[i]);
    std::copy(rc_w[i].begin(), rc_w[i].end(), f->fw.begin() + f->fo[i]);
  }
  std::vector<int32_t> cnt(n_active, 0);
  for (int64_t i = 0; i < nnz; ++i) cnt[f->fc[i]]++;
  f->ao.assign(n_active + 1, 0);
  int32_t off = 0;
  for (int32_t i = 0; i < n_active; ++i) {
    f->ao[i] = off;
    off += cnt[i];
  }
  f->ao[n_active] = off;
  f->ac.resize(nnz);
  f->aw.resize(nnz);
  std::vector<int32_t> cur(f->ao.begin(), f->ao.end() - 1);
  for (int32_t r = 0; r < n_active; ++r)
    for (int32_t k = f->fo[r]; k < f->fo[r + 1]; ++k) {
      int32_t t = cur[f->fc[k]]++;
      f->ac[t] = r;
      f->aw[t] = f->fw[k];
    }
  f->s.assign(n_active, 0.0);
  for (int32_t i = 0; i < n_active; ++i) {
    double s = 0.0;
    for (int32_t k = f->ao[i]; k < f->ao[i + 1]; ++k) s += f->aw[k];
    f->s[i] = s;
  }
  return f;
}

extern "C" void orc_filter_free(orc_filter* f) { delete f; }
extern "C" int64_t orc_filter_nnz(const orc_filter* f) { return (int64_t)f->fc.size(); }
extern "C" void orc_filter_s(const orc_filter* f, double* out) { std::copy(f->s.begin(), f->s.end(), out); }

extern "C" void orc_filter_apply(const orc_filter* f, const double* in, double* out) {
#pragma omp parallel for schedule(static)
  for (int32_t r = 0; r < f->n; ++r) {
    double s = 0.0;
    for (int32_t k = f->fo[r]; k < f->fo[r + 1]; ++k) s += f->fw[k] * in[f->fc[k]];
    out[r] = s;
  }
}

extern "C" void orc_filter_adjoint(const orc_filter* f, const double* in, double* out) {
#pragma omp parallel for schedule(static)
  for (int32_t r = 0; r < f->n; ++r) {
    double s = 0.0;
    for (int32_t k = f->ao[r]; k < f->ao[r + 1]; ++k) s += f->aw[k] * in[f->ac[k]];
    out[r] = s;
  }
}

// ---------------------------------------------------------------------------------------------------------
// SensitivityAnalysis — src/Mycel.Core/Optimization/SensitivityAnalysis.cs:13-146
// ---------------------------------------------------------------------------------------------------------
extern "C" void orc_sensitivities(orc_op* op, const double* u, const double* rho, double* dc, double penal) {
  orc_model* m = op->m;
  double dE = m->e0 - m->emin;
  int64_t na = (int64_t)m->active_elements.size();
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < na; ++k) {
    int32_t dofs[24];
    double ue[24];
    element_dofs(m, m->active_elements[k], dofs);
    for (int i = 0; i < 24; ++i) ue[i] = u[dofs[i]];
    double se = 0.0;
    for (int r = 0; r < 24; ++r) {
      double s = 0.0;
      for (int c = 0; c < 24; ++c) s += op->ke[r * 24 + c] * ue[c];
      se += ue[r] * s;
    }
    double dEdr = penal * mpow(rho[k], penal - 1.0) * dE;
    dc[k] = -dEdr * se;
  }
}

// ---------------------------------------------------------------------------------------------------------
// OcOptimizer — src/Mycel.Core/Optimization/OcOptimizer.cs:12-175
// ---------------------------------------------------------------------------------------------------------
namespace {
inline double clampd(double v, double lo, double hi) {  // Math.Clamp(double)
  if (v < lo) return lo;
  if (v > hi) return hi;
  return v;
}
inline double maxd(double a, double b) {  // Math.Max(double): NaN propagates
  if (std::isnan(a) || std::isnan(b)) return NAN;
  return a > b ? a : b;
}
inline double mind(double a, double b) {
  if (std::isnan(a) || std::isnan(b)) return NAN;
  return a < b ? a : b;
}

double eval_volume(const double* rho, const double* dc, const double* s, const uint8_t* pas, int32_t n, double lam,
                   double move, double rmin) {
  double vol = 0.0;
  for (int32_t i = 0; i < n; ++i) {
    if (pas && pas[i]) {
      vol += s[i] * 1.0;
      continue;
    }
    double r = rho[i], si = s[i];
    double lo = maxd(rmin, r - move), hi = mind(1.0, r + move);
    double nd = -dc[i];
    if (nd <= 0.0 || si <= 0.0) vol += si * lo;
    else {
      double b = nd / (lam * si);
      vol += si * clampd(r * std::sqrt(b), lo, hi);
    }
  }
  return vol;
}
}  // namespace

namespace {
// OcOptimizer.Update; trace (optional) records each volume evaluation's lambda and V(lambda) in order.
double oc_update_impl(const double* rho, const double* dc, const double* s, const uint8_t* pas, double* rho_new,
                      int32_t n, double f, double move, double rmin, double lg, int32_t maxb, double voltol,
                      std::vector<double>* trace) {
  double ts = 0.0;
  for (int32_t i = 0; i < n; ++i) ts += s[i];
  double tv = f * ts;
  auto vol = [&](double lam) {
    double v = eval_volume(rho, dc, s, pas, n, lam, move, rmin);
    if (trace) {
      trace->push_back(lam);
      trace->push_back(v);
    }
    return v;
  };
  bool ok = lg > 0.0 && !std::isinf(lg) && !std::isnan(lg);
  double l1 = ok ? lg * 0.5 : 1e-12;
  double l2 = ok ? lg * 2.0 : 1e12;
  if (l1 <= 1e-50) l1 = 1e-12;
  if (l2 <= l1) l2 = l1 * 10.0;
  double v1 = vol(l1);
  double v2 = vol(l2);
  int ex = 0;
  while (v1 < tv && l1 > 1e-50 && ex++ < 50) {
    l2 = l1;
    v2 = v1;
    l1 *= 0.1;
    v1 = vol(l1);
  }
  ex = 0;
  while (v2 > tv && l2 < 1e50 && ex++ < 50) {
    l1 = l2;
    v1 = v2;
    l2 *= 10.0;
    v2 = vol(l2);
  }
  double lm = std::sqrt(l1 * l2);
  for (int32_t st = 0; st < maxb; ++st) {
    lm = std::sqrt(l1 * l2);
    double vm = vol(lm);
    double re = std::fabs(vm - tv) / maxd(tv, 1e-12);
    if (re <= voltol) break;
    if (vm > tv) l1 = lm;
    else l2 = lm;
    if (std::fabs(l2 - l1) <= 1e-15 * lm) break;
  }
  for (int32_t i = 0; i < n; ++i) {
    if (pas && pas[i]) {
      rho_new[i] = 1.0;
      continue;
    }
    double r = rho[i], si = s[i];
    double lo = maxd(rmin, r - move), hi = mind(1.0, r + move);
    double nd = -dc[i];
    if (nd <= 0.0 || si <= 0.0) rho_new[i] = lo;
    else {
      double b = nd / (lm * si);
      rho_new[i] = clampd(r * std::sqrt(b), lo, hi);
    }
  }
  return lm;
}
}  // namespace

extern "C" double orc_oc_update(const double* rho, const double* dc, const double* s, const uint8_t* pas,
                                double* rho_new, int32_t n, double f, double move, double rmin, double lg,
                                int32_t maxb, double voltol) {
  return oc_update_impl(rho, dc, s, pas, rho_new, n, f, move, rmin, lg, maxb, voltol, nullptr);
}

extern "C" int32_t orc_oc_trace(const double* rho, const double* dc, const double* s, const uint8_t* pas, int32_t n,
                                double f, double move, double rmin, double lg, int32_t maxb, double voltol,
                                double* lam_out, double* vol_out, int32_t cap, double* total_s_out) {
  std::vector<double> rn((size_t)std::max(n, 1)), tr;
  oc_update_impl(rho, dc, s, pas, rn.data(), n, f, move, rmin, lg, maxb, voltol, &tr);
  double ts = 0.0;
  for (int32_t i = 0; i < n; ++i) ts += s[i];
  if (total_s_out) *total_s_out = ts;
  int32_t cnt = (int32_t)(tr.size() / 2);
  for (int32_t k = 0; k < cnt && k < cap; ++k) {
    lam_out[k] = tr[2 * k];
    vol_out[k] = tr[2 * k + 1];
  }
  return cnt;
}

// HeavisideProjection (HeavisideProjection.cs:12-37)
extern "C" void orc_heaviside_project(const double* rt, double* rb, int32_t n, double beta, double eta) {
  double den = std::tanh(beta * eta) + std::tanh(beta * (1.0 - eta));
  double inv = 1.0 / den;
  double tbe = std::tanh(beta * eta);
  for (int32_t i = 0; i < n; ++i) rb[i] = clampd((tbe + std::tanh(beta * (rt[i] - eta))) * inv, 0.0, 1.0);
}
extern "C" void orc_heaviside_derivative(const double* rt, double* d, int32_t n, double beta, double eta) {
  double den = std::tanh(beta * eta) + std::tanh(beta * (1.0 - eta));
  double inv = 1.0 / den;
  for (int32_t i = 0; i < n; ++i) {
    double t = std::tanh(beta * (rt[i] - eta));
    d[i] = maxd(beta * (1.0 - t * t) * inv, 1e-12);
  }
}

// PassiveRegion.Build (src/Mycel.Core/Voxelization/PassiveRegion.cs:13-62)
extern "C" void orc_passive_region(int nx, int ny, int nz, const int32_t* nodes, int32_t nn, int rad, uint8_t* out) {
  std::memset(out, 0, (size_t)nx * ny * nz);
  int nx1 = nx + 1, ny1 = ny + 1;
  for (int32_t q = 0; q < nn; ++q) {
    int n = nodes[q];
    int nk = n / (nx1 * ny1), rem = n % (nx1 * ny1), nj = rem / nx1, ni = rem % nx1;
    auto cl = [](int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); };
    int x0 = cl(ni - rad, 0, nx - 1), x1 = cl(ni + rad - 1, 0, nx - 1);
    int y0 = cl(nj - rad, 0, ny - 1), y1 = cl(nj + rad - 1, 0, ny - 1);
    int z0 = cl(nk - rad, 0, nz - 1), z1 = cl(nk + rad - 1, 0, nz - 1);
    for (int iz = z0; iz <= z1; ++iz)
      for (int iy = y0; iy <= y1; ++iy)
        for (int ix = x0; ix <= x1; ++ix) out[ix + nx * (iy + ny * iz)] = 1;
  }
}

// ---------------------------------------------------------------------------------------------------------
// TopologyOptimizer.Run — src/Mycel.Core/Optimization/TopologyOptimizer.cs:16-407
// ---------------------------------------------------------------------------------------------------------
extern "C" int orc_topopt_run(orc_model* m, const orc_simp_options* o, orc_iter_record* hist, int32_t cap,
                              int32_t* n_iters, int32_t* converged_out, double* u_out, float* phys_out,
                              float* design_out, double* rho_phys_active, double* rho_design_active,
                              double* lambda_out, char* msg, int msglen) {
  *n_iters = 0;
  *converged_out = 0;
  double h = (double)m->h;
  double f = o->volume_fraction;
  double rmin = o->filter_radius_mm / h;
  if (rmin < 1.5 && o->enforce_min_filter_radius) rmin = 1.5;
  int32_t na = (int32_t)m->active_elements.size();
  const std::vector<int32_t>& act = m->active_elements;
  int64_t te = m->total_elements;
  std::vector<uint8_t> pas(na, 0);
  if (o->passive_mask)
    for (int32_t i = 0; i < na; ++i)
      if (act[i] < o->passive_len && o->passive_mask[act[i]] != 0) pas[i] = 1;
  if (o->protect_boundary_hinges) {
    std::vector<int32_t> pn;
    std::unordered_set<int32_t> seen;
    for (const orc_load& l : m->loads)
      for (int32_t nd : l.nodes)
        if (seen.insert(nd).second) pn.push_back(nd);
    for (int32_t d : m->fixed)
      if (seen.insert(d / 3).second) pn.push_back(d / 3);
    std::vector<uint8_t> shell(te);
    orc_passive_region(m->nx, m->ny, m->nz, pn.data(), (int32_t)pn.size(), 1, shell.data());
    for (int32_t i = 0; i < na; ++i)
      if (shell[act[i]]) pas[i] = 1;
  }
  orc_filter* filt = orc_filter_create(m->nx, m->ny, m->nz, m->domain.data(), act.data(), na, rmin);
  std::vector<double> s(na);
  orc_filter_s(filt, s.data());
  std::vector<double> rho(na);
  if (o->initial_density) {
    if (o->initial_density_len == te) {
      for (int32_t i = 0; i < na; ++i) rho[i] = (double)o->initial_density[act[i]];
    } else if (o->initial_density_len == na) {
      for (int32_t i = 0; i < na; ++i) rho[i] = (double)o->initial_density[i];
    } else {
      orc_filter_free(filt);
      set_msg(msg, msglen, "InitialDensity length must match either TotalElements or ActiveElementCount.");
      return ORC_E_ARG;
    }
  } else {
    for (int32_t i = 0; i < na; ++i) rho[i] = pas[i] ? 1.0 : f;
  }
  for (int32_t i = 0; i < na; ++i)
    if (pas[i]) rho[i] = 1.0;
  std::vector<double> rt(na), rb(na), rold(na), dcb(na), dct, dd, dc(na);
  if (o->enable_heaviside) {
    dct.resize(na);
    dd.resize(na);
  }
  int64_t nd = m->total_dofs;
  std::vector<double> u(nd, 0.0);
  if (o->warm_start && o->warm_start_len == nd) std::copy(o->warm_start, o->warm_start + nd, u.begin());
  orc_op* op = orc_op_create(m);
  // Load cases: summed into one right-hand side as the reference does, or (separate_load_cases) kept apart:
  // one solve per case with its own warm start, compliance sum_k F_k.u_k and sensitivities summed over the
  // cases in case order (objective sum_k c_k, an extension: the reference has no multi-load objective)
  const int ncase = o->separate_load_cases ? std::max<int>(1, (int)m->loads.size()) : 1;
  std::vector<std::vector<double>> Fk(ncase, std::vector<double>(nd)), bk(ncase, std::vector<double>(nd));
  std::vector<std::vector<double>> uk;
  int st = ORC_OK;
  for (int k = 0; k < ncase && !st; ++k)
    st = o->separate_load_cases && !m->loads.empty() ? orc_model_assemble_case_forces(m, k, Fk[k].data(), msg, msglen)
                                                     : orc_model_assemble_forces(m, Fk[k].data(), msg, msglen);
  if (st) {
    orc_op_free(op);
    orc_filter_free(filt);
    return st;
  }
  for (int k = 0; k < ncase; ++k)
    for (int64_t i = 0; i < nd; ++i) bk[k][i] = m->constrained[i] ? 0.0 : Fk[k][i];
  if (o->separate_load_cases) uk.assign(ncase, std::vector<double>(nd, 0.0));
  std::vector<double> dck(o->separate_load_cases ? na : 0);
  double lambda = 1.0, maxChange = 1.0, beta = 1.0;
  int conv = 0;
  std::vector<double> chist;
  int start = o->start_iteration, maxit = o->max_iterations;
  double pbase = o->penal;
  int count = 0;
  double rpcg_first = 0;
  (void)rpcg_first;
  for (int iter = start; iter <= maxit; ++iter) {
    double penal = pbase;
    if (o->continuation) penal = iter < 20 ? 1.0 : (iter < 40 ? 2.0 : pbase);
    for (int32_t i = 0; i < na; ++i)
      if (pas[i]) rho[i] = 1.0;
    if (o->enable_heaviside) {
      orc_filter_apply(filt, rho.data(), rt.data());
      orc_heaviside_project(rt.data(), rb.data(), na, beta, 0.5);
    } else {
      orc_filter_apply(filt, rho.data(), rb.data());
    }
    for (int32_t i = 0; i < na; ++i) m->density[act[i]] = rb[i];
    orc_op_update_densities(op, m->density.data(), penal);
    double tol;
    if (iter == start) tol = o->solver_tol_initial;
    else {
      double ta = clampd((maxChange - 0.01) / 0.09, 0.0, 1.0);
      double li = std::log10(maxd(o->solver_tol_initial, 1e-15));
      double lf = std::log10(maxd(o->solver_tol_final, 1e-15));
      double lt = lf + ta * (li - lf);
      tol = std::pow(10.0, lt);
    }
    orc_pcg_result pr;
    int iters = 0;
    double resid = 0.0, c = 0.0, md = 0.0;
    for (int k = 0; k < ncase; ++k) {
      std::vector<double>& uc = o->separate_load_cases ? uk[k] : u;
      st = orc_pcg_solve(op, bk[k].data(), uc.data(), tol, o->solver_max_iterations, &pr, msg, msglen);
      if (st) break;
      if (!pr.converged) {
        char buf[400];
        std::snprintf(buf, sizeof buf,
                      "FEM solver did not converge in %d iterations (%s). Is the model not sufficiently constrained?",
                      pr.iterations, pr.message);
        set_msg(msg, msglen, buf);
        st = ORC_E_NOT_CONVERGED;
        break;
      }
      iters += pr.iterations;
      resid = std::max(resid, pr.final_residual);
      double ck = 0.0;
      for (int64_t i = 0; i < nd; ++i) ck += Fk[k][i] * uc[i];
      c += ck;
      for (int64_t q = 0; q < m->total_nodes; ++q)
        if (m->active_nodes[q]) {
          double ux = uc[3 * q], uy = uc[3 * q + 1], uz = uc[3 * q + 2];
          double sq = ux * ux + uy * uy + uz * uz;
          if (sq > md) md = sq;
        }
      if (k == 0) {
        orc_sensitivities(op, uc.data(), rb.data(), dcb.data(), penal);
      } else {
        orc_sensitivities(op, uc.data(), rb.data(), dck.data(), penal);
        for (int32_t i = 0; i < na; ++i) dcb[i] = dcb[i] + dck[i];
      }
    }
    if (st) break;
    md = std::sqrt(md);
    if (o->separate_load_cases) {  // u reported: the superposition sum_k u_k, in case order
      for (int64_t i = 0; i < nd; ++i) u[i] = uk[0][i];
      for (int k = 1; k < ncase; ++k)
        for (int64_t i = 0; i < nd; ++i) u[i] = u[i] + uk[k][i];
    }
    if (o->enable_heaviside) {
      orc_heaviside_derivative(rt.data(), dd.data(), na, beta, 0.5);
      for (int32_t i = 0; i < na; ++i) dct[i] = dcb[i] * dd[i];
      orc_filter_adjoint(filt, dct.data(), dc.data());
    } else {
      orc_filter_adjoint(filt, dcb.data(), dc.data());
    }
    rold = rho;
    lambda = orc_oc_update(rho.data(), dc.data(), s.data(), pas.data(), rho.data(), na, f, o->move_limit, o->rho_min,
                           lambda, 60, 1e-8);
    if (o->enable_heaviside && iter % 25 == 0 && beta < 8.0) beta = std::min(8.0, beta * 2.0);
    maxChange = 0.0;
    double cv = 0.0, gs = 0.0;
    for (int32_t i = 0; i < na; ++i) {
      double d = std::fabs(rho[i] - rold[i]);
      if (d > maxChange) maxChange = d;
      cv += rb[i];
      double r = o->enable_heaviside ? rt[i] : rb[i];
      gs += r * (1.0 - r);
    }
    if (count < cap) {
      orc_iter_record& rec = hist[count];
      rec.iteration = iter;
      rec.compliance = c;
      rec.volume_fraction = cv / na;
      rec.max_change = maxChange;
      rec.grey_level = (4.0 * gs / na) * 100.0;
      rec.solver_iterations = iters;
      rec.solver_residual = resid;
      rec.max_displacement = md;
      rec.total_ms = 0;
    }
    ++count;
    if (phys_out) {
      for (int64_t e = 0; e < te; ++e) phys_out[e] = 0.0f;
      for (int32_t i = 0; i < na; ++i) phys_out[act[i]] = (float)rb[i];
    }
    if (design_out) {
      for (int64_t e = 0; e < te; ++e) design_out[e] = 0.0f;
      for (int32_t i = 0; i < na; ++i) design_out[act[i]] = (float)rho[i];
    }
    if (rho_phys_active) std::copy(rb.begin(), rb.end(), rho_phys_active);
    if (rho_design_active) std::copy(rho.begin(), rho.end(), rho_design_active);
    chist.push_back(c);
    if (chist.size() > 6) chist.erase(chist.begin());
    if (chist.size() == 6) {
      double rc = std::fabs(c - chist.front()) / c;
      if (maxChange < 0.01 && rc < 1e-3) {
        conv = 1;
        break;
      }
    }
  }
  *n_iters = count;
  *converged_out = conv;
  if (lambda_out) *lambda_out = lambda;
  if (u_out) std::copy(u.begin(), u.end(), u_out);
  orc_op_free(op);
  orc_filter_free(filt);
  return st;
}

// ---------------------------------------------------------------------------------------------------------
extern "C" void orc_set_lane_mode(int mode) { g_lane_mode = mode; }
extern "C" void orc_math_pow(int64_t n, const double* x, const double* y, int64_t y_len, double* out) {
  for (int64_t i = 0; i < n; ++i) out[i] = mpow(x[i], y[y_len == 1 ? 0 : i]);
}
extern "C" void orc_set_threads(int n) {
#ifdef _OPENMP
  omp_set_num_threads(n > 0 ? n : 1);
#else
  (void)n;
#endif
}
extern "C" int orc_get_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

// ---------------------------------------------------------------------------------------------------------
// RunWriter.ComputeQuantizedChecksum (src/Mycel.Core/Persistence/RunWriter.cs:344-356) and the quantisation of
// WriteIterationFileAtomic (:211-217): q = (byte)MathF.Round(Math.Clamp(v, 0, 1) * 255f, AwayFromZero); FNV-1a
// 32-bit over the bytes in order (offset basis 2166136261, prime 16777619). Writes q when out is non-NULL.
extern "C" uint32_t orc_quantized_checksum(const float* v, int64_t n, uint8_t* out) {
  uint32_t h = 2166136261u;
  for (int64_t i = 0; i < n; ++i) {
    float c = v[i] < 0.0f ? 0.0f : (v[i] > 1.0f ? 1.0f : v[i]);
    float x = c * 255.0f;
    uint8_t q = (uint8_t)std::round(x);  // std::round: half away from zero, like MidpointRounding.AwayFromZero
    if (out) out[i] = q;
    h ^= q;
    h *= 16777619u;
  }
  return h;
}

// ---------------------------------------------------------------------------------------------------------
// SurfaceNetsExtractor.Extract (src/Mycel.Core/PostProcessing/SurfaceNetsExtractor.cs:31-312), with
// MakeWellComposed (:352-435), Resolve2x2Saddle (:437-451), Resolve3DCornerKiss (:453-476) and EmitQuad
// (:314-346). Sequential, in the reference's loop orders; float arithmetic with every operation rounded
// (no contraction), as RyuJIT evaluates the Vector3 expressions. Vector3.DistanceSquared is taken as
// (dx*dx + dy*dy) + dz*dz and Vector3 / float as a component-wise division.
// ---------------------------------------------------------------------------------------------------------
struct orc_mesh {
  std::vector<float> pos;     // 3 per vertex
  std::vector<int32_t> idx;   // 3 per triangle
  int32_t passes = 0;         // well-composedness passes run
  int64_t changes = 0;        // saddle and corner-kiss resolutions made
};

namespace {

bool sn_saddle(std::vector<uint8_t>& s, std::vector<float>& rho, float thr, int64_t i00, int64_t i10, int64_t i01,
               int64_t i11) {
  const bool s00 = s[i00], s10 = s[i10], s01 = s[i01], s11 = s[i11];
  if (!(s00 == s11 && s10 == s01 && s00 != s10)) return false;
  const int64_t a = s00 ? i10 : i00, b = s00 ? i01 : i11;  // the two empty voxels of the diagonal pair
  const int64_t pick = rho[a] >= rho[b] ? a : b;
  s[pick] = 1;
  if (rho[pick] < thr) rho[pick] = thr;
  return true;
}

bool sn_kiss(std::vector<uint8_t>& s, std::vector<float>& rho, float thr, int64_t dA, int64_t dB, int64_t a1,
             int64_t a2, int64_t a3, int64_t b1, int64_t b2, int64_t b3) {
  if (!(s[dA] && s[dB])) return false;
  const bool linked = (s[a1] && (s[b1] || s[b2])) || (s[a2] && (s[b1] || s[b3])) || (s[a3] && (s[b2] || s[b3]));
  if (linked) return false;
  s[a1] = 1;
  s[b1] = 1;
  if (rho[a1] < thr) rho[a1] = thr;
  if (rho[b1] < thr) rho[b1] = thr;
  return true;
}

}  // namespace

extern "C" orc_mesh* orc_surface_nets(int nx, int ny, int nz, float h, const float* origin, const float* density,
                                      float thr) {
  orc_mesh* m = new orc_mesh();
  const int64_t PX = nx + 2, PY = ny + 2, PZ = nz + 2, SY = PX, SZ = PX * PY;
  std::vector<float> rho((size_t)(PX * PY * PZ), 0.0f);
  std::vector<uint8_t> sol((size_t)(PX * PY * PZ), 0);
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        const float v = density[x + (int64_t)nx * (y + (int64_t)ny * z)];
        const int64_t p = (x + 1) + SY * (y + 1) + SZ * (z + 1);
        rho[p] = v;
        sol[p] = v >= thr;
      }
  // well-composedness: face saddles, then corner kisses, until a pass changes nothing (at most 8 passes)
  bool changed = true;
  while (changed && m->passes < 8) {
    changed = false;
    m->passes++;
    for (int64_t z = 1; z <= nz; ++z)
      for (int64_t y = 1; y <= ny; ++y)
        for (int64_t x = 1; x <= nx; ++x) {
          const int64_t b = x + y * SY + z * SZ;
          if (x < nx && y < ny && sn_saddle(sol, rho, thr, b, b + 1, b + SY, b + SY + 1)) changed = true, m->changes++;
          if (x < nx && z < nz && sn_saddle(sol, rho, thr, b, b + 1, b + SZ, b + SZ + 1)) changed = true, m->changes++;
          if (y < ny && z < nz && sn_saddle(sol, rho, thr, b, b + SY, b + SZ, b + SZ + SY)) changed = true, m->changes++;
        }
    for (int64_t z = 1; z < nz; ++z)
      for (int64_t y = 1; y < ny; ++y)
        for (int64_t x = 1; x < nx; ++x) {
          const int64_t c000 = x + y * SY + z * SZ, c100 = c000 + 1, c010 = c000 + SY, c110 = c000 + SY + 1;
          const int64_t c001 = c000 + SZ, c101 = c001 + 1, c011 = c001 + SY, c111 = c001 + SY + 1;
          if (sn_kiss(sol, rho, thr, c000, c111, c100, c010, c001, c110, c101, c011) ||
              sn_kiss(sol, rho, thr, c100, c011, c000, c110, c101, c010, c001, c111) ||
              sn_kiss(sol, rho, thr, c010, c101, c000, c110, c011, c100, c001, c111) ||
              sn_kiss(sol, rho, thr, c001, c110, c000, c101, c011, c100, c010, c111))
            changed = true, m->changes++;
        }
  }
  // one vertex per dual cell with mixed corners, in cell order (cz, cy, cx)
  static const int edges[12][2] = {{0, 1}, {2, 3}, {4, 5}, {6, 7}, {0, 2}, {1, 3},
                                   {4, 6}, {5, 7}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};
  const int64_t CX = nx + 1, CY = ny + 1, CZ = nz + 1;
  std::vector<int32_t> vidx((size_t)(CX * CY * CZ), -1);
  for (int64_t cz = 0; cz < CZ; ++cz)
    for (int64_t cy = 0; cy < CY; ++cy)
      for (int64_t cx = 0; cx < CX; ++cx) {
        float cr[8];
        bool cs[8];
        int mask = 0;
        for (int c = 0; c < 8; ++c) {
          const int64_t p = (cx + (c & 1)) + SY * (cy + ((c >> 1) & 1)) + SZ * (cz + (c >> 2));
          cr[c] = rho[p];
          cs[c] = sol[p];
          if (cs[c]) mask |= 1 << c;
        }
        if (mask == 0 || mask == 255) continue;
        float sx = 0.f, sy = 0.f, sz = 0.f;
        int cnt = 0;
        for (int e = 0; e < 12; ++e) {
          const int a = edges[e][0], b = edges[e][1];
          if (cs[a] == cs[b]) continue;
          const float va = cr[a], vb = cr[b];
          const float den = vb - va;
          float al = 0.5f;
          if (std::fabs(den) > 1e-12f) {
            al = (thr - va) / den;
            al = al < 0.05f ? 0.05f : (al > 0.95f ? 0.95f : al);
          }
          const float oa[3] = {(a & 1) - 0.5f, ((a >> 1) & 1) - 0.5f, (a >> 2) - 0.5f};
          const float ob[3] = {(b & 1) - 0.5f, ((b >> 1) & 1) - 0.5f, (b >> 2) - 0.5f};
          const float px = oa[0] + al * (ob[0] - oa[0]);
          const float py = oa[1] + al * (ob[1] - oa[1]);
          const float pz = oa[2] + al * (ob[2] - oa[2]);
          sx = sx + px;
          sy = sy + py;
          sz = sz + pz;
          cnt++;
        }
        float ox = 0.f, oy = 0.f, oz = 0.f;
        if (cnt > 0) {
          const float fc = (float)cnt;
          ox = sx / fc;
          oy = sy / fc;
          oz = sz / fc;
        }
        vidx[(size_t)(cx + CX * (cy + CY * cz))] = (int32_t)(m->pos.size() / 3);
        m->pos.push_back(origin[0] + ((float)cx + ox) * h);
        m->pos.push_back(origin[1] + ((float)cy + oy) * h);
        m->pos.push_back(origin[2] + ((float)cz + oz) * h);
      }
  if (m->pos.empty()) return m;
  auto cell = [&](int64_t x, int64_t y, int64_t z) { return vidx[(size_t)(x + CX * (y + CY * z))]; };
  auto d2 = [&](int32_t i, int32_t j) {
    const float dx = m->pos[3 * i] - m->pos[3 * j], dy = m->pos[3 * i + 1] - m->pos[3 * j + 1],
                dz = m->pos[3 * i + 2] - m->pos[3 * j + 2];
    const float xx = dx * dx, yy = dy * dy, zz = dz * dz;
    return (xx + yy) + zz;
  };
  auto quad = [&](int32_t v0, int32_t v1, int32_t v2, int32_t v3, bool flip) {
    if (v0 < 0 || v1 < 0 || v2 < 0 || v3 < 0) return;
    if (flip) std::swap(v1, v3);
    if (d2(v0, v2) <= d2(v1, v3)) {
      m->idx.insert(m->idx.end(), {v0, v1, v2, v0, v2, v3});
    } else {
      m->idx.insert(m->idx.end(), {v0, v1, v3, v1, v2, v3});
    }
  };
  for (int64_t z = 1; z <= nz; ++z)  // x-directed grid edges
    for (int64_t y = 1; y <= ny; ++y)
      for (int64_t x = 0; x <= nx; ++x) {
        const bool s0 = sol[x + y * SY + z * SZ], s1 = sol[x + 1 + y * SY + z * SZ];
        if (s0 != s1) quad(cell(x, y - 1, z - 1), cell(x, y, z - 1), cell(x, y, z), cell(x, y - 1, z), !s0);
      }
  for (int64_t z = 1; z <= nz; ++z)  // y-directed
    for (int64_t y = 0; y <= ny; ++y)
      for (int64_t x = 1; x <= nx; ++x) {
        const bool s0 = sol[x + y * SY + z * SZ], s1 = sol[x + (y + 1) * SY + z * SZ];
        if (s0 != s1) quad(cell(x - 1, y, z - 1), cell(x - 1, y, z), cell(x, y, z), cell(x, y, z - 1), !s0);
      }
  for (int64_t z = 0; z <= nz; ++z)  // z-directed
    for (int64_t y = 1; y <= ny; ++y)
      for (int64_t x = 1; x <= nx; ++x) {
        const bool s0 = sol[x + y * SY + z * SZ], s1 = sol[x + y * SY + (z + 1) * SZ];
        if (s0 != s1) quad(cell(x - 1, y - 1, z), cell(x, y - 1, z), cell(x, y, z), cell(x - 1, y, z), !s0);
      }
  return m;
}

extern "C" void orc_mesh_info(const orc_mesh* m, int64_t* out) {
  out[0] = (int64_t)(m->pos.size() / 3);
  out[1] = (int64_t)m->idx.size();
  out[2] = m->passes;
  out[3] = m->changes;
}
extern "C" void orc_mesh_copy(const orc_mesh* m, float* pos, int32_t* idx) {
  std::copy(m->pos.begin(), m->pos.end(), pos);
  std::copy(m->idx.begin(), m->idx.end(), idx);
}
extern "C" void orc_mesh_free(orc_mesh* m) { delete m; }

// StaticAnalysis.AverageElementToNode (src/Mycel.Core/Fem/StaticAnalysis.cs:222-268): node sums in the active
// element order, then sum / count.
extern "C" void orc_average_element_to_node(const orc_model* m, const double* es, double* out) {
  const int64_t nx1 = m->nx + 1, ny1 = m->ny + 1;
  std::vector<double> sum((size_t)m->total_nodes, 0.0);
  std::vector<int> cnt((size_t)m->total_nodes, 0);
  for (int32_t e : m->active_elements) {
    const int64_t ix = e % m->nx, iy = (e / m->nx) % m->ny, iz = e / ((int64_t)m->nx * m->ny);
    const int64_t n0 = ix + nx1 * (iy + ny1 * iz), n1 = n0 + 1, n3 = n0 + nx1, n2 = n3 + 1;
    const int64_t n4 = n0 + nx1 * ny1, n5 = n4 + 1, n7 = n4 + nx1, n6 = n7 + 1;
    const int64_t ns[8] = {n0, n1, n2, n3, n4, n5, n6, n7};
    for (int64_t q : ns) {
      sum[(size_t)q] += es[e];
      cnt[(size_t)q]++;
    }
  }
  for (int64_t q = 0; q < m->total_nodes; ++q) out[q] = cnt[(size_t)q] > 0 ? sum[(size_t)q] / cnt[(size_t)q] : 0.0;
}

// TaubinSmoother.Smooth (src/Mycel.Core/PostProcessing/TaubinSmoother.cs:15-101, ApplyLaplacianStep :103-134):
// per vertex the sorted, de-duplicated neighbours over all triangles; each iteration a +lambda then a mu
// Laplacian step, p + (factor / count) * sum(q - p) with every Vector3 operation rounded per component.
extern "C" void orc_taubin_smooth(float* pos, int64_t nv, const int32_t* idx, int64_t ni, int iterations, float lambda,
                                  float mu) {
  if (iterations <= 0 || nv == 0 || ni < 3) return;
  std::vector<std::vector<int32_t>> nb((size_t)nv);
  for (int64_t t = 0; t + 2 < ni; t += 3) {
    const int32_t a = idx[t], b = idx[t + 1], c = idx[t + 2];
    nb[a].push_back(b); nb[a].push_back(c);
    nb[b].push_back(c); nb[b].push_back(a);
    nb[c].push_back(a); nb[c].push_back(b);
  }
  for (int64_t v = 0; v < nv; ++v) {
    auto& l = nb[(size_t)v];
    if (l.empty()) continue;
    std::sort(l.begin(), l.end());
    std::vector<int32_t> u;
    u.push_back(l[0]);
    for (size_t k = 1; k < l.size(); ++k)
      if (l[k] != u.back() && l[k] != (int32_t)v) u.push_back(l[k]);
    l.swap(u);
  }
  std::vector<float> cur(pos, pos + 3 * nv), tmp((size_t)(3 * nv));
  auto step = [&](const std::vector<float>& src, std::vector<float>& dst, float factor) {
    for (int64_t v = 0; v < nv; ++v) {
      const auto& l = nb[(size_t)v];
      const float px = src[3 * v], py = src[3 * v + 1], pz = src[3 * v + 2];
      if (l.empty()) {
        dst[3 * v] = px; dst[3 * v + 1] = py; dst[3 * v + 2] = pz;
        continue;
      }
      float sx = 0.f, sy = 0.f, sz = 0.f;
      for (int32_t q : l) {
        sx = sx + (src[3 * (size_t)q] - px);
        sy = sy + (src[3 * (size_t)q + 1] - py);
        sz = sz + (src[3 * (size_t)q + 2] - pz);
      }
      const float w = factor / (float)l.size();
      dst[3 * v] = px + w * sx;
      dst[3 * v + 1] = py + w * sy;
      dst[3 * v + 2] = pz + w * sz;
    }
  };
  for (int it = 0; it < iterations; ++it) {
    step(cur, tmp, lambda);
    step(tmp, cur, mu);
  }
  std::copy(cur.begin(), cur.end(), pos);
}
