// ORACLE -- test infrastructure only (never shipped, never on the product path).
//
// FP64 CPU restatement of DDHDG's per-cell HDG kernel for structured Cartesian
// meshes (quads / hexes / segments, axis-aligned, uniform spacing):
//   * cell quadrature data           include/assembling_methods.template.h:134-265
//   * cc volume terms                include/assembling_methods.template.h:269-532
//   * cc_rhs volume terms            include/assembling_methods.template.h:536-760
//   * face quadrature data           include/assembling_methods.template.h:764-820
//   * ct                             include/assembling_methods.template.h:885-1019
//   * ct -> cc_rhs                   include/assembling_methods.template.h:1023-1141
//   * tc                             include/assembling_methods.template.h:1145-1307
//   * tc -> tt_rhs                   include/assembling_methods.template.h:1311-1447
//   * tt                             include/assembling_methods.template.h:1451-1547
//   * tt -> tt_rhs                   include/assembling_methods.template.h:1551-1588
//   * Dirichlet L2 projection        include/assembling_methods.template.h:1592-1691
//   * Neumann                        include/assembling_methods.template.h:1695-1734
//   * border terms                   include/assembling_methods.template.h:1737-2118
//   * trace terms (reconstruction)   include/assembling_methods.template.h:2122-2160
//   * boundary flux dispatch         include/assembling_methods.template.h:2164-2286
//   * per-cell driver + Schur        include/assembling_methods.template.h:2290-2698
//   * Dirichlet column condensation  src/local_condenser.cpp:142-160
//   * SRH / linear recombination     src/recombination_term.cpp:116-160,433-575
//   * quasi Fermi potential          include/solver.h:343-376
// The loops run over every enabled cell dof for every quadrature point exactly
// like the reference (structural zeros included), and the local inverse is an
// explicit LU-based inverse like FullMatrix::gauss_jordan (getrf+getri for
// n > 15).  This file is also the timed CPU baseline (OpenMP over cells, the
// analogue of WorkStream).
//
// Finite elements (deal.II 9, not vendored): FE_DGQ(k) and FE_FaceQ(k) are
// tensor-product Lagrange bases on Gauss-Lobatto support points (a single
// constant function for k = 0); quadrature is QGauss(k+1) on cells and faces.
// Cell dof order inside one cell follows the FESystem
//   [ E_0..E_{d-1}, V, Wn_0..Wn_{d-1}, n, Wp_0..Wp_{d-1}, p ] x (k+1)^d nodes
// and the restricted trace order is [face][enabled component][face node].

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace
{
  constexpr double KB = 1.380649E-23;
  constexpr double Q  = 1.602176634E-19;
  constexpr double EV = 1.602176565E-19;

  enum Flux
  {
    USE_CELL  = 0,
    USE_TRACE = 1,
    QIU_SHI   = 2
  };
} // namespace

extern "C"
{
  // Flat problem description.  All arrays are owned by the caller.
  struct OrProblem
  {
    int    dim, k;
    int    n[3];
    double origin[3];
    double h[3];
    int    enabled[3];
    int    flux;
    int    phi_linearize;
    int    rec_type; // 0: linear recombination, 1: SRH with fixed temperature
    double eps;      // rescaled permittivity
    double mu_n, mu_p;
    double temperature;
    double thermal_voltage_rescale;
    double V_rescale, n_rescale, rec_rescale;
    double nc, nv, ec_eV, ev_eV;
    double srh_ni, srh_tau_n, srh_tau_p;
    const double *rec_a, *rec_b, *rec_c; // [ncells*nqc] (may be null -> 0)
    const double *doping;                // [ncells*nqc] rescaled doping
    const double *tau;                   // [ncells*2*dim*3] rescaled tau
    const int    *face_bc;               // [nfaces*3]: 0 none, 1 Dirichlet, 2 Neumann
    const double *face_bc_val;           // [nfaces*3*nqf] already rescaled
    // Jacobian options; 0 reproduces the reference exactly.
    //  bit 0: consistent sign of the E coupling of the cell drift terms
    //  bit 1: recombination derivatives scaled by the doping magnitude
    int jacobian_fix;
  };
}

namespace
{
  // ---------------------------------------------------------------- 1D tools
  double
  legendre(int n, double x, double *dp)
  {
    double p0 = 1., p1 = x, d0 = 0., d1 = 1.;
    if (n == 0)
      {
        if (dp)
          *dp = 0.;
        return 1.;
      }
    for (int i = 2; i <= n; ++i)
      {
        const double p2 = ((2. * i - 1.) * x * p1 - (i - 1.) * p0) / i;
        const double d2 = d0 + (2. * i - 1.) * p1;
        p0 = p1;
        p1 = p2;
        d0 = d1;
        d1 = d2;
      }
    if (dp)
      *dp = d1;
    return p1;
  }

  // Gauss-Legendre rule with m points on [0,1] (QGauss<1>(m)).
  void
  gauss_rule(int m, std::vector<double> &x, std::vector<double> &w)
  {
    x.resize(m);
    w.resize(m);
    for (int i = 0; i < m; ++i)
      {
        double t = std::cos(M_PI * (i + 0.75) / (m + 0.5));
        for (int it = 0; it < 100; ++it)
          {
            double       d;
            const double p  = legendre(m, t, &d);
            const double dt = p / d;
            t -= dt;
            if (std::fabs(dt) < 1e-16)
              break;
          }
        double d;
        legendre(m, t, &d);
        // ascending order on [0,1]
        x[m - 1 - i] = 0.5 * (1. + t);
        w[m - 1 - i] = 1. / ((1. - t * t) * d * d);
      }
  }

  // Gauss-Lobatto support points with k+1 points on [0,1]; midpoint for k=0.
  std::vector<double>
  lobatto_points(int k)
  {
    std::vector<double> x(k + 1);
    if (k == 0)
      {
        x[0] = 0.5;
        return x;
      }
    x[0] = 0.;
    x[k] = 1.;
    for (int i = 1; i < k; ++i)
      {
        // interior points: roots of P'_k on (-1,1)
        double t = -std::cos(M_PI * i / k);
        for (int it = 0; it < 200; ++it)
          {
            // f = P'_k(t); f' = P''_k(t) = (2 t P'_k - k(k+1) P_k)/(1-t^2)
            double       d;
            const double p   = legendre(k, t, &d);
            const double dd  = (2. * t * d - k * (k + 1.) * p) / (1. - t * t);
            const double del = d / dd;
            t -= del;
            if (std::fabs(del) < 1e-16)
              break;
          }
        x[i] = 0.5 * (1. + t);
      }
    std::sort(x.begin(), x.end());
    return x;
  }

  struct Lagrange1D
  {
    std::vector<double> nodes;
    double
    val(int a, double x) const
    {
      double r = 1.;
      for (int b = 0; b < (int)nodes.size(); ++b)
        if (b != a)
          r *= (x - nodes[b]) / (nodes[a] - nodes[b]);
      return r;
    }
    double
    der(int a, double x) const
    {
      double s = 0.;
      for (int m = 0; m < (int)nodes.size(); ++m)
        {
          if (m == a)
            continue;
          double r = 1. / (nodes[a] - nodes[m]);
          for (int b = 0; b < (int)nodes.size(); ++b)
            if (b != a && b != m)
              r *= (x - nodes[b]) / (nodes[a] - nodes[b]);
          s += r;
        }
      return s;
    }
  };

  // --------------------------------------------------------- tiny vectors
  struct Vec
  {
    double v[3] = {0., 0., 0.};
  };
  inline double
  dot(const Vec &a, const Vec &b, int d)
  {
    double s = 0.;
    for (int i = 0; i < d; ++i)
      s += a.v[i] * b.v[i];
    return s;
  }
  inline Vec
  scale(const Vec &a, double s)
  {
    Vec r;
    for (int i = 0; i < 3; ++i)
      r.v[i] = a.v[i] * s;
    return r;
  }

  // ---------------------------------------------------- geometry tables
  struct Geometry
  {
    int dim, k, nb, nf, nqc, nqf, nfaces_cell;
    int n[3];
    long ncells, nfaces;
    long axis_face_offset[4];
    double h[3], origin[3];

    std::vector<double> g1, w1;          // Gauss rule
    Lagrange1D          cellb, faceb;    // GL Lagrange bases
    // cell tables
    std::vector<double> cphi;   // [nqc][nb]
    std::vector<Vec>    cgrad;  // [nqc][nb] (physical)
    std::vector<double> cJxW;   // [nqc]
    std::vector<Vec>    cqref;  // [nqc] reference coordinates
    // face tables, per local face f
    std::vector<double> fphi;   // [F][nqf][nb] cell basis on face
    std::vector<double> fxi;    // [nqf][nf]    trace basis
    std::vector<double> fJxW;   // [F][nqf]
    std::vector<Vec>    fnormal;// [F]
    std::vector<Vec>    fqref;  // [F][nqf] reference coordinates in the cell

    void
    init(const OrProblem &P)
    {
      dim = P.dim;
      k   = P.k;
      nb  = 1;
      nf  = 1;
      for (int i = 0; i < dim; ++i)
        nb *= (k + 1);
      for (int i = 0; i < dim - 1; ++i)
        nf *= (k + 1);
      nqc         = nb;
      nqf         = nf;
      nfaces_cell = 2 * dim;
      ncells      = 1;
      for (int a = 0; a < 3; ++a)
        {
          n[a]      = (a < dim) ? P.n[a] : 1;
          h[a]      = (a < dim) ? P.h[a] : 1.;
          origin[a] = (a < dim) ? P.origin[a] : 0.;
          ncells *= n[a];
        }
      long off = 0;
      for (int a = 0; a < dim; ++a)
        {
          axis_face_offset[a] = off;
          long cnt            = 1;
          for (int b = 0; b < dim; ++b)
            cnt *= (b == a) ? (n[b] + 1) : n[b];
          off += cnt;
        }
      axis_face_offset[dim] = off;
      nfaces                = off;

      gauss_rule(k + 1, g1, w1);
      cellb.nodes = lobatto_points(k);
      faceb.nodes = lobatto_points(k);

      double vol = 1.;
      for (int a = 0; a < dim; ++a)
        vol *= h[a];

      cphi.assign(nqc * nb, 0.);
      cgrad.assign(nqc * nb, Vec());
      cJxW.assign(nqc, 0.);
      cqref.assign(nqc, Vec());
      for (int q = 0; q < nqc; ++q)
        {
          int qi[3] = {0, 0, 0};
          int r     = q;
          for (int a = 0; a < dim; ++a)
            {
              qi[a] = r % (k + 1);
              r /= (k + 1);
            }
          double w = vol;
          for (int a = 0; a < dim; ++a)
            {
              w *= w1[qi[a]];
              cqref[q].v[a] = g1[qi[a]];
            }
          cJxW[q] = w;
          for (int i = 0; i < nb; ++i)
            {
              int ai[3] = {0, 0, 0};
              int rr    = i;
              for (int a = 0; a < dim; ++a)
                {
                  ai[a] = rr % (k + 1);
                  rr /= (k + 1);
                }
              double v = 1.;
              for (int a = 0; a < dim; ++a)
                v *= cellb.val(ai[a], g1[qi[a]]);
              cphi[q * nb + i] = v;
              for (int s = 0; s < dim; ++s)
                {
                  double g = 1.;
                  for (int a = 0; a < dim; ++a)
                    g *= (a == s) ? cellb.der(ai[a], g1[qi[a]]) / h[a] :
                                    cellb.val(ai[a], g1[qi[a]]);
                  cgrad[q * nb + i].v[s] = g;
                }
            }
        }

      fphi.assign(nfaces_cell * nqf * nb, 0.);
      fxi.assign(nqf * nf, 0.);
      fJxW.assign(nfaces_cell * nqf, 0.);
      fnormal.assign(nfaces_cell, Vec());
      fqref.assign(nfaces_cell * nqf, Vec());
      for (int qf = 0; qf < nqf; ++qf)
        {
          int qi[2] = {0, 0};
          int r     = qf;
          for (int t = 0; t < dim - 1; ++t)
            {
              qi[t] = r % (k + 1);
              r /= (k + 1);
            }
          for (int m = 0; m < nf; ++m)
            {
              int mi[2] = {0, 0};
              int rr    = m;
              for (int t = 0; t < dim - 1; ++t)
                {
                  mi[t] = rr % (k + 1);
                  rr /= (k + 1);
                }
              double v = 1.;
              for (int t = 0; t < dim - 1; ++t)
                v *= faceb.val(mi[t], g1[qi[t]]);
              fxi[qf * nf + m] = v;
            }
        }
      for (int f = 0; f < nfaces_cell; ++f)
        {
          const int a    = f / 2;
          const int side = f % 2;
          fnormal[f].v[a] = side ? 1. : -1.;
          double area     = 1.;
          for (int b = 0; b < dim; ++b)
            if (b != a)
              area *= h[b];
          for (int qf = 0; qf < nqf; ++qf)
            {
              int qi[2] = {0, 0};
              int r     = qf;
              for (int t = 0; t < dim - 1; ++t)
                {
                  qi[t] = r % (k + 1);
                  r /= (k + 1);
                }
              Vec    xr;
              double w = area;
              xr.v[a]  = side ? 1. : 0.;
              for (int t = 0; t < dim - 1; ++t)
                {
                  const int ax = (a + 1 + t) % dim;
                  xr.v[ax]     = g1[qi[t]];
                  w *= w1[qi[t]];
                }
              fJxW[f * nqf + qf]  = w;
              fqref[f * nqf + qf] = xr;
              for (int i = 0; i < nb; ++i)
                {
                  int ai[3] = {0, 0, 0};
                  int rr    = i;
                  for (int b = 0; b < dim; ++b)
                    {
                      ai[b] = rr % (k + 1);
                      rr /= (k + 1);
                    }
                  double v = 1.;
                  for (int b = 0; b < dim; ++b)
                    v *= cellb.val(ai[b], xr.v[b]);
                  fphi[(f * nqf + qf) * nb + i] = v;
                }
            }
        }
    }

    void
    cell_index(long c, int ci[3]) const
    {
      ci[0] = c % n[0];
      ci[1] = (c / n[0]) % n[1];
      ci[2] = c / ((long)n[0] * n[1]);
    }

    long
    face_of_cell(long c, int f) const
    {
      int ci[3];
      cell_index(c, ci);
      const int a = f / 2;
      int       fi[3] = {ci[0], ci[1], ci[2]};
      fi[a] += f % 2;
      long idx = 0, stride = 1;
      for (int b = 0; b < dim; ++b)
        {
          const int extent = (b == a) ? n[b] + 1 : n[b];
          idx += fi[b] * stride;
          stride *= extent;
        }
      return axis_face_offset[a] + idx;
    }

    // does cell basis function i (node index) have support on local face f
    bool
    node_on_face(int i, int f) const
    {
      if (k == 0)
        return true;
      const int a    = f / 2;
      const int side = f % 2;
      int       rr   = i;
      int       ai   = 0;
      for (int b = 0; b <= a; ++b)
        {
          ai = rr % (k + 1);
          rr /= (k + 1);
        }
      return side ? (ai == k) : (ai == 0);
    }
  };

  // -------------------------------------------------------- dense helpers
  // Explicit inverse through LU with partial pivoting of the matrix handed
  // over as-is (getrf + getri on the array).
  bool
  invert_lu(std::vector<double> &A, int n)
  {
    std::vector<int>    piv(n);
    std::vector<double> LU = A;
    for (int j = 0; j < n; ++j)
      {
        int    p  = j;
        double mx = std::fabs(LU[j * n + j]);
        for (int i = j + 1; i < n; ++i)
          if (std::fabs(LU[i * n + j]) > mx)
            {
              mx = std::fabs(LU[i * n + j]);
              p  = i;
            }
        piv[j] = p;
        if (mx == 0.)
          return false;
        if (p != j)
          for (int c = 0; c < n; ++c)
            std::swap(LU[j * n + c], LU[p * n + c]);
        const double inv = 1. / LU[j * n + j];
        for (int i = j + 1; i < n; ++i)
          {
            const double l = LU[i * n + j] * inv;
            LU[i * n + j]  = l;
            if (l != 0.)
              for (int c = j + 1; c < n; ++c)
                LU[i * n + c] -= l * LU[j * n + c];
          }
      }
    // solve LU X = P I column by column
    std::vector<double> col(n);
    for (int c = 0; c < n; ++c)
      {
        std::fill(col.begin(), col.end(), 0.);
        col[c] = 1.;
        for (int j = 0; j < n; ++j)
          if (piv[j] != j)
            std::swap(col[j], col[piv[j]]);
        for (int i = 0; i < n; ++i)
          {
            double s = col[i];
            for (int j = 0; j < i; ++j)
              s -= LU[i * n + j] * col[j];
            col[i] = s;
          }
        for (int i = n - 1; i >= 0; --i)
          {
            double s = col[i];
            for (int j = i + 1; j < n; ++j)
              s -= LU[i * n + j] * col[j];
            col[i] = s / LU[i * n + i];
          }
        for (int i = 0; i < n; ++i)
          A[i * n + c] = col[i];
      }
    return true;
  }

  // Gauss-Jordan in place with row interchanges (Stoer & Bulirsch), the
  // algorithm FullMatrix::gauss_jordan runs itself for n <= 15.
  bool
  invert_gauss_jordan(std::vector<double> &A, int n)
  {
    std::vector<int> p(n);
    for (int i = 0; i < n; ++i)
      p[i] = i;
    for (int j = 0; j < n; ++j)
      {
        double max = std::fabs(A[j * n + j]);
        int    r   = j;
        for (int i = j + 1; i < n; ++i)
          if (std::fabs(A[i * n + j]) > max)
            {
              max = std::fabs(A[i * n + j]);
              r   = i;
            }
        if (max == 0.)
          return false;
        if (r > j)
          {
            for (int k = 0; k < n; ++k)
              std::swap(A[j * n + k], A[r * n + k]);
            std::swap(p[j], p[r]);
          }
        const double hr = 1. / A[j * n + j];
        A[j * n + j]    = hr;
        for (int k = 0; k < n; ++k)
          {
            if (k == j)
              continue;
            for (int i = 0; i < n; ++i)
              {
                if (i == j)
                  continue;
                A[i * n + k] -= A[i * n + j] * A[j * n + k] * hr;
              }
          }
        for (int i = 0; i < n; ++i)
          {
            A[i * n + j] *= hr;
            A[j * n + i] *= -hr;
          }
        A[j * n + j] = hr;
      }
    std::vector<double> hv(n);
    for (int i = 0; i < n; ++i)
      {
        for (int k = 0; k < n; ++k)
          hv[p[k]] = A[i * n + k];
        for (int k = 0; k < n; ++k)
          A[i * n + k] = hv[k];
      }
    return true;
  }

  // FullMatrix::gauss_jordan: for n > 15 deal.II hands its row-major storage
  // to LAPACK getrf/getri, which read it as the transpose; the inverse of the
  // transpose read back row-major is the inverse.  The LU therefore pivots
  // along the rows of the matrix, which makes it insensitive to the very
  // different row scales of the V block (rescaled permittivity) and the flux
  // blocks.  Smaller matrices use the in-place Gauss-Jordan above.
  bool
  invert(std::vector<double> &A, int n)
  {
    if (n <= 15)
      return invert_gauss_jordan(A, n);
    std::vector<double> T(n * n);
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j)
        T[j * n + i] = A[i * n + j];
    if (!invert_lu(T, n))
      return false;
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j)
        A[i * n + j] = T[j * n + i];
    return true;
  }

  // Cholesky solve of a small SPD system (LAPACKFullMatrix::compute_cholesky)
  void
  cholesky_solve(std::vector<double> &M, std::vector<double> &b, int n)
  {
    for (int j = 0; j < n; ++j)
      {
        double s = M[j * n + j];
        for (int c = 0; c < j; ++c)
          s -= M[j * n + c] * M[j * n + c];
        s            = std::sqrt(s);
        M[j * n + j] = s;
        for (int i = j + 1; i < n; ++i)
          {
            double t = M[i * n + j];
            for (int c = 0; c < j; ++c)
              t -= M[i * n + c] * M[j * n + c];
            M[i * n + j] = t / s;
          }
      }
    for (int i = 0; i < n; ++i)
      {
        double s = b[i];
        for (int c = 0; c < i; ++c)
          s -= M[i * n + c] * b[c];
        b[i] = s / M[i * n + i];
      }
    for (int i = n - 1; i >= 0; --i)
      {
        double s = b[i];
        for (int c = i + 1; c < n; ++c)
          s -= M[c * n + i] * b[c];
        b[i] = s / M[i * n + i];
      }
  }

  // ------------------------------------------------------------ the kernel
  struct Outputs
  {
    // non-null entries are filled
    double *cc, *ct, *tc, *tt, *cc_rhs, *tt_rhs; // local system (Schur or not)
    int    *dbc_local;                           // [Nt] 1 if Dirichlet dof
    double *dbc_value;                           // [Nt]
    double *update_cell;                         // [Nc_all] (reconstruction)
  };

  struct Workspace
  {
    // per-dof shape data at the current qp, indexed by enabled dof
    std::vector<Vec>    d[3];
    std::vector<double> d_div[3], c[3];
    std::vector<Vec>    c_grad[3];
    std::vector<double> trc[3]; // trace shape values (by face-local index)
    std::vector<double> cc, ct, tc, tt, cc_rhs, tt_rhs, tmp;
  };

  class Oracle
  {
  public:
    Oracle(const OrProblem &P)
      : P(P)
    {
      G.init(P);
      dim       = G.dim;
      nb        = G.nb;
      nf        = G.nf;
      Nc_all    = 3 * (dim + 1) * nb;
      ncomp_en  = 0;
      for (int c = 0; c < 3; ++c)
        if (P.enabled[c])
          comp_index[c] = ncomp_en++;
        else
          comp_index[c] = -1;
      Nt = G.nfaces_cell * ncomp_en * nf;
      for (int i = 0; i < Nc_all; ++i)
        if (P.enabled[i / ((dim + 1) * nb)])
          enabled_dofs.push_back(i);
      Nc = (int)enabled_dofs.size();
      // cell support on face: positions into enabled_dofs
      cell_on_face.resize(G.nfaces_cell);
      for (int f = 0; f < G.nfaces_cell; ++f)
        for (int i = 0; i < Nc; ++i)
          if (G.node_on_face(enabled_dofs[i] % nb, f))
            cell_on_face[f].push_back(i);
      // trace support on face: local trace dofs of face f
      trace_on_face.resize(G.nfaces_cell);
      for (int f = 0; f < G.nfaces_cell; ++f)
        for (int i = 0; i < ncomp_en * nf; ++i)
          trace_on_face[f].push_back(f * ncomp_en * nf + i);
    }

    const OrProblem &P;
    Geometry         G;
    int              dim, nb, nf, Nc_all, Nc, Nt, ncomp_en;
    int              comp_index[3];
    std::vector<int> enabled_dofs;
    std::vector<std::vector<int>> cell_on_face, trace_on_face;

    // value of the displacement / scalar of component blk for enabled dof i
    inline void
    shape_cell(int q, int i, int blk, Vec &dv, double &ddiv, double &cv,
               Vec &cg) const
    {
      const int dof = enabled_dofs[i];
      const int b   = dof / ((dim + 1) * nb);
      const int sub = (dof / nb) % (dim + 1);
      const int a   = dof % nb;
      dv            = Vec();
      ddiv          = 0.;
      cv            = 0.;
      cg            = Vec();
      if (b != blk)
        return;
      if (sub < dim)
        {
          dv.v[sub] = G.cphi[q * nb + a];
          ddiv      = G.cgrad[q * nb + a].v[sub];
        }
      else
        {
          cv = G.cphi[q * nb + a];
          cg = G.cgrad[q * nb + a];
        }
    }

    inline void
    shape_face(int f, int qf, int i, int blk, Vec &dv, double &cv) const
    {
      const int dof = enabled_dofs[i];
      const int b   = dof / ((dim + 1) * nb);
      const int sub = (dof / nb) % (dim + 1);
      const int a   = dof % nb;
      dv            = Vec();
      cv            = 0.;
      if (b != blk)
        return;
      const double v = G.fphi[(f * G.nqf + qf) * nb + a];
      if (sub < dim)
        dv.v[sub] = v;
      else
        cv = v;
    }

    // value of trace shape function (restricted local index) of component
    // blk at face qp qf of local face f
    inline double
    shape_trace(int f, int qf, int lt, int blk) const
    {
      const int face = lt / (ncomp_en * nf);
      if (face != f)
        return 0.;
      const int ce = (lt / nf) % ncomp_en;
      if (ce != comp_index[blk])
        return 0.;
      return G.fxi[qf * nf + lt % nf];
    }

    // previous cell values at a point (cell reference coords by table)
    void
    eval_cell_fields(const double *coef, const double *phi,
                     double cval[3], Vec dval[3]) const
    {
      for (int b = 0; b < 3; ++b)
        {
          cval[b] = 0.;
          dval[b] = Vec();
          for (int s = 0; s <= dim; ++s)
            {
              double acc = 0.;
              for (int a = 0; a < nb; ++a)
                acc += coef[(b * (dim + 1) + s) * nb + a] * phi[a];
              if (s < dim)
                dval[b].v[s] = acc;
              else
                cval[b] = acc;
            }
        }
    }

    void
    recombination(double n, double p, long cell, int q, double &r,
                  double &drn, double &drp) const
    {
      const double rf = P.n_rescale;
      if (P.rec_type == 1)
        {
          const double ni  = P.srh_ni / rf;
          const double tn  = P.srh_tau_n;
          const double tp  = P.srh_tau_p;
          const double num = n * p - ni * ni;
          const double den = tp * (n + ni) + tn * (p + ni);
          r                = num * rf / den;
          drn              = p / den - num * tp / (den * den);
          drp              = n / den - num * tn / (den * den);
        }
      else
        {
          const long   idx = cell * G.nqc + q;
          const double a   = P.rec_a ? P.rec_a[idx] : 0.;
          const double b   = P.rec_b ? P.rec_b[idx] : 0.;
          const double c   = P.rec_c ? P.rec_c[idx] : 0.;
          r                = a + (b * n + c * p) * rf;
          drn              = b;
          drp              = c;
        }
      r /= P.rec_rescale;
      drn /= P.rec_rescale;
      drp /= P.rec_rescale;
      if (P.jacobian_fix & 2)
        {
          // d(R/R_s)/d(n/N) = N dR/dn / R_s; the reference omits the N
          drn *= rf;
          drp *= rf;
        }
    }

    double
    qf_potential(int comp, double density, double potential, double T) const
    {
      const double U_T = T * (KB / Q);
      if (comp == 1)
        return potential - P.ec_eV * EV / Q - U_T * std::log(density / P.nc);
      return potential - P.ev_eV * EV / Q + U_T * std::log(density / P.nv);
    }

    // The per-cell worker.  reconstruct: update_trace is the full trace
    // update [nfaces][3][nf].
    void
    cell_system(long cell, const double *cell_state, const double *trace_state,
                const double *update_trace, bool reconstruct, bool thermo,
                bool schur, Workspace &w, Outputs &out) const
    {
      const int    nqc = G.nqc, nqf = G.nqf;
      const bool   Ven = P.enabled[0], nen = P.enabled[1], pen = P.enabled[2];
      const bool   phi_mode = P.phi_linearize || thermo;
      const double *coef    = cell_state + cell * Nc_all;

      w.cc.assign(Nc * Nc, 0.);
      w.cc_rhs.assign(Nc, 0.);
      if (!reconstruct)
        {
          w.ct.assign(Nc * Nt, 0.);
          w.tc.assign(Nt * Nc, 0.);
          w.tt.assign(Nt * Nt, 0.);
          w.tt_rhs.assign(Nt, 0.);
        }
      std::vector<int>    cons_dof;
      std::vector<double> cons_val;

      const double U_T = (KB * P.temperature / Q) / P.thermal_voltage_rescale;
      const double eps = P.eps, mun = P.mu_n, mup = P.mu_p;
      const double drift_sign = (P.jacobian_fix & 1) ? -1. : 1.;

      // ---- prepare_data_on_cell_quadrature_points (T:134-265)
      std::vector<double> V0(nqc), n0(nqc), p0(nqc), rr(nqc, 0.), drn(nqc, 0.),
        drp(nqc, 0.), phin(nqc, 0.), phip(nqc, 0.), C(nqc, 0.);
      std::vector<Vec> E0(nqc), Wn0(nqc), Wp0(nqc);
      for (int q = 0; q < nqc; ++q)
        {
          double cv[3];
          Vec    dv[3];
          eval_cell_fields(coef, &G.cphi[q * nb], cv, dv);
          V0[q]  = cv[0];
          n0[q]  = cv[1];
          p0[q]  = cv[2];
          E0[q]  = dv[0];
          Wn0[q] = dv[1];
          Wp0[q] = dv[2];
          if (Ven)
            C[q] = P.doping[cell * nqc + q];
          if (nen || pen)
            recombination(n0[q], p0[q], cell, q, rr[q], drn[q], drp[q]);
          if (P.phi_linearize)
            {
              if (nen)
                phin[q] = qf_potential(1, n0[q] * P.n_rescale,
                                       V0[q] * P.V_rescale, P.temperature);
              if (pen)
                phip[q] = qf_potential(2, p0[q] * P.n_rescale,
                                       V0[q] * P.V_rescale, P.temperature);
            }
        }

      const double nc = P.nc, nv = P.nv, ec = P.ec_eV * EV, ev = P.ev_eV * EV;
      const double V_rescale = P.V_rescale, n_rescale = P.n_rescale;

      // ---- add_cell_products_to_cc_matrix (T:269-532)
      std::vector<Vec>    dd[3], cg[3];
      std::vector<double> ddiv[3], cvv[3];
      for (int b = 0; b < 3; ++b)
        {
          dd[b].resize(Nc);
          cg[b].resize(Nc);
          ddiv[b].resize(Nc);
          cvv[b].resize(Nc);
        }
      for (int q = 0; q < nqc; ++q)
        {
          const double JxW = G.cJxW[q];
          for (int i = 0; i < Nc; ++i)
            for (int b = 0; b < 3; ++b)
              shape_cell(q, i, b, dd[b][i], ddiv[b][i], cvv[b][i], cg[b][i]);

          const Vec mun_E0 = scale(E0[q], mun);
          const Vec mup_E0 = scale(E0[q], mup);

          double phi_V_der = 0.;
          if (phi_mode)
            {
              const double KbT_over_q  = KB * P.temperature / (Q * V_rescale);
              const double ev_rescaled = ev / (Q * V_rescale);
              const double ec_rescaled = ec / (Q * V_rescale);
              const double phn = thermo ? 0. : phin[q] / V_rescale;
              const double php = thermo ? 0. : phip[q] / V_rescale;
              phi_V_der =
                -1 / n_rescale *
                (nv / KbT_over_q *
                   std::exp((ev_rescaled - V0[q] + php) / KbT_over_q) +
                 nc / KbT_over_q *
                   std::exp((V0[q] - phn - ec_rescaled) / KbT_over_q));
            }

          for (int i = 0; i < Nc; ++i)
            for (int j = 0; j < Nc; ++j)
              {
                double s = 0.;
                if (Ven)
                  {
                    const Vec eps_E = scale(dd[0][j], eps);
                    s += (-cvv[0][j] * ddiv[0][i] + dot(dd[0][j], dd[0][i], dim) -
                          dot(eps_E, cg[0][i], dim)) *
                         JxW;
                    if (phi_mode)
                      s += -phi_V_der * cvv[0][j] * cvv[0][i] * JxW;
                    else
                      s += (cvv[1][j] - cvv[2][j]) * cvv[0][i] * JxW;
                  }
                if (nen)
                  {
                    const Vec mun_E   = scale(dd[0][j], mun);
                    const Vec Dn_Wn   = scale(scale(dd[1][j], mun), U_T);
                    // the reference adds +n0 (mu E_j . grad z) here although
                    // the residual's derivative is -n0 (mu dE . grad z)
                    s += (-cvv[1][j] * ddiv[1][i] + dot(dd[1][j], dd[1][i], dim) -
                          cvv[1][j] * dot(mun_E0, cg[1][i], dim) +
                          drift_sign * n0[q] * dot(mun_E, cg[1][i], dim) +
                          dot(Dn_Wn, cg[1][i], dim) -
                          (drn[q] * cvv[1][j] + drp[q] * cvv[2][j]) * cvv[1][i]) *
                         JxW;
                  }
                if (pen)
                  {
                    const Vec mup_E = scale(dd[0][j], mup);
                    const Vec Dp_Wp = scale(scale(dd[2][j], mup), U_T);
                    s += (-cvv[2][j] * ddiv[2][i] + dot(dd[2][j], dd[2][i], dim) +
                          cvv[2][j] * dot(mup_E0, cg[2][i], dim) -
                          drift_sign * p0[q] * dot(mup_E, cg[2][i], dim) +
                          dot(Dp_Wp, cg[2][i], dim) -
                          (drn[q] * cvv[1][j] + drp[q] * cvv[2][j]) * cvv[2][i]) *
                         JxW;
                  }
                w.cc[i * Nc + j] += s;
              }

          // ---- add_cell_products_to_cc_rhs (T:536-760)
          Vec    Jn, Jp;
          double phi_rhs = 0.;
          if (nen)
            {
              const Vec DWn = scale(scale(Wn0[q], mun), U_T);
              for (int a = 0; a < 3; ++a)
                Jn.v[a] = n0[q] * mun_E0.v[a] - DWn.v[a];
            }
          if (pen)
            {
              const Vec DWp = scale(scale(Wp0[q], mup), U_T);
              for (int a = 0; a < 3; ++a)
                Jp.v[a] = -p0[q] * mup_E0.v[a] - DWp.v[a];
            }
          if (phi_mode)
            {
              const double KbT_over_q  = KB * P.temperature / (Q * V_rescale);
              const double ev_rescaled = ev / (Q * V_rescale);
              const double ec_rescaled = ec / (Q * V_rescale);
              const double phn = thermo ? 0. : phin[q] / V_rescale;
              const double php = thermo ? 0. : phip[q] / V_rescale;
              phi_rhs =
                1 / n_rescale *
                (nv * std::exp((ev_rescaled - V0[q] + php) / KbT_over_q) -
                 nc * std::exp((V0[q] - phn - ec_rescaled) / KbT_over_q));
            }
          const Vec eps_E0 = scale(E0[q], eps);
          for (int i = 0; i < Nc; ++i)
            {
              double s = 0.;
              if (Ven)
                {
                  s += (V0[q] * ddiv[0][i] - dot(E0[q], dd[0][i], dim) +
                        dot(eps_E0, cg[0][i], dim) + C[q] * cvv[0][i]) *
                       JxW;
                  if (phi_mode)
                    s += phi_rhs * cvv[0][i] * JxW;
                  else
                    s += (-n0[q] + p0[q]) * cvv[0][i] * JxW;
                }
              if (nen)
                s += (n0[q] * ddiv[1][i] - dot(Wn0[q], dd[1][i], dim) +
                      rr[q] * cvv[1][i] + dot(Jn, cg[1][i], dim)) *
                     JxW;
              if (pen)
                s += (p0[q] * ddiv[2][i] - dot(Wp0[q], dd[2][i], dim) +
                      rr[q] * cvv[2][i] + dot(Jp, cg[2][i], dim)) *
                     JxW;
              w.cc_rhs[i] += s;
            }
        }

      // does the cell touch any boundary condition (T:2701-2748)
      bool has_bc = false;
      for (int f = 0; f < G.nfaces_cell; ++f)
        {
          const long F = G.face_of_cell(cell, f);
          for (int b = 0; b < 3; ++b)
            if (P.enabled[b] && P.face_bc[F * 3 + b] != 0)
              has_bc = true;
        }

      // ---- faces
      std::vector<Vec>    fdv[3];
      std::vector<double> fcv[3];
      for (int b = 0; b < 3; ++b)
        {
          fdv[b].resize(Nc);
          fcv[b].resize(Nc);
        }
      for (int f = 0; f < G.nfaces_cell; ++f)
        {
          const long F      = G.face_of_cell(cell, f);
          const Vec &normal = G.fnormal[f];
          // prepare_data_on_face_quadrature_points (T:764-820)
          std::vector<double> c0f[3], trc0[3], dtr[3], tauf[3];
          std::vector<Vec>    d0f[3];
          for (int b = 0; b < 3; ++b)
            {
              c0f[b].assign(nqf, 0.);
              trc0[b].assign(nqf, 0.);
              dtr[b].assign(nqf, 0.);
              d0f[b].assign(nqf, Vec());
              tauf[b].assign(nqf, P.tau[(cell * G.nfaces_cell + f) * 3 + b]);
            }
          for (int qf = 0; qf < nqf; ++qf)
            {
              double cv[3];
              Vec    dv[3];
              eval_cell_fields(coef, &G.fphi[(f * nqf + qf) * nb], cv, dv);
              for (int b = 0; b < 3; ++b)
                {
                  c0f[b][qf] = cv[b];
                  d0f[b][qf] = dv[b];
                  double t = 0., u = 0.;
                  for (int m = 0; m < nf; ++m)
                    {
                      t += trace_state[(F * 3 + b) * nf + m] * G.fxi[qf * nf + m];
                      if (update_trace)
                        u += update_trace[(F * 3 + b) * nf + m] *
                             G.fxi[qf * nf + m];
                    }
                  trc0[b][qf] = t;
                  dtr[b][qf]  = u;
                }
            }
          const double U_Tf = U_T;

          // ---- add_ct_matrix_terms_to_cc_rhs (T:1023-1141)
          for (int qf = 0; qf < nqf; ++qf)
            {
              const double JxW = G.fJxW[f * nqf + qf];
              for (int ii : cell_on_face[f])
                {
                  double s = 0.;
                  Vec    qv;
                  double zv;
                  if (Ven)
                    {
                      shape_face(f, qf, ii, 0, qv, zv);
                      s += (-trc0[0][qf] * dot(qv, normal, dim) +
                            tauf[0][qf] * trc0[0][qf] * zv) *
                           JxW;
                    }
                  if (nen)
                    {
                      shape_face(f, qf, ii, 1, qv, zv);
                      s += (-trc0[1][qf] * dot(qv, normal, dim) -
                            tauf[1][qf] * trc0[1][qf] * zv) *
                           JxW;
                    }
                  if (pen)
                    {
                      shape_face(f, qf, ii, 2, qv, zv);
                      s += (-trc0[2][qf] * dot(qv, normal, dim) -
                            tauf[2][qf] * trc0[2][qf] * zv) *
                           JxW;
                    }
                  w.cc_rhs[ii] += s;
                }
            }

          if (!reconstruct)
            {
              // ---- assemble_ct_matrix (T:885-1019)
              for (int qf = 0; qf < nqf; ++qf)
                {
                  const double JxW = G.fJxW[f * nqf + qf];
                  const double E0n = dot(d0f[0][qf], normal, dim);
                  const Vec    mun_E0 = scale(d0f[0][qf], mun);
                  const Vec    mup_E0 = scale(d0f[0][qf], mup);
                  for (int i : cell_on_face[f])
                    {
                      Vec    q1, q2, q3;
                      double z1, z2, z3;
                      shape_face(f, qf, i, 0, q1, z1);
                      shape_face(f, qf, i, 1, q2, z2);
                      shape_face(f, qf, i, 2, q3, z3);
                      for (int j : trace_on_face[f])
                        {
                          double s = 0.;
                          if (Ven)
                            {
                              const double trV = shape_trace(f, qf, j, 0);
                              s += (trV * dot(q1, normal, dim) -
                                    tauf[0][qf] * trV * z1) *
                                   JxW;
                            }
                          if (nen)
                            {
                              const double trn = shape_trace(f, qf, j, 1);
                              if (P.flux == USE_TRACE ||
                                  (P.flux == QIU_SHI && E0n <= 0))
                                s += dot(mun_E0, normal, dim) * trn * z2 * JxW;
                              s += (trn * dot(q2, normal, dim) +
                                    tauf[1][qf] * (trn * z2)) *
                                   JxW;
                            }
                          if (pen)
                            {
                              const double trp = shape_trace(f, qf, j, 2);
                              if (P.flux == USE_TRACE ||
                                  (P.flux == QIU_SHI && E0n <= 0))
                                s += -dot(mup_E0, normal, dim) * trp * z3 * JxW;
                              s += (trp * dot(q3, normal, dim) +
                                    tauf[2][qf] * (trp * z3)) *
                                   JxW;
                            }
                          w.ct[i * Nt + j] += s;
                        }
                    }
                }

              // ---- per component: Dirichlet or tc/tt (+Neumann)
              for (int b = 0; b < 3; ++b)
                {
                  if (!P.enabled[b])
                    continue;
                  const int bc = has_bc ? P.face_bc[F * 3 + b] : 0;
                  if (bc == 1)
                    {
                      // apply_dbc_on_face (T:1592-1691)
                      std::vector<int> dofs;
                      for (int j : trace_on_face[f])
                        if ((j / nf) % ncomp_en == comp_index[b])
                          dofs.push_back(j);
                      const int           m = (int)dofs.size();
                      std::vector<double> M(m * m, 0.), rhs(m, 0.);
                      for (int qf = 0; qf < nqf; ++qf)
                        {
                          const double JxW = G.fJxW[f * nqf + qf];
                          const double val =
                            thermo ? 0. :
                                     P.face_bc_val[(F * 3 + b) * nqf + qf] -
                                       trc0[b][qf];
                          for (int i = 0; i < m; ++i)
                            {
                              const double bi = G.fxi[qf * nf + dofs[i] % nf];
                              for (int j = 0; j < m; ++j)
                                M[i * m + j] +=
                                  bi * G.fxi[qf * nf + dofs[j] % nf] * JxW;
                              rhs[i] += bi * val * JxW;
                            }
                        }
                      cholesky_solve(M, rhs, m);
                      for (int i = 0; i < m; ++i)
                        {
                          cons_dof.push_back(dofs[i]);
                          cons_val.push_back(rhs[i]);
                        }
                      continue;
                    }
                  // assemble_tc_matrix (T:1145-1307)
                  for (int qf = 0; qf < nqf; ++qf)
                    {
                      const double JxW = G.fJxW[f * nqf + qf];
                      const double E0n = dot(d0f[0][qf], normal, dim);
                      const Vec    mu_E0 =
                        scale(d0f[0][qf], b == 1 ? mun : mup);
                      const double mu = (b == 1) ? mun : mup;
                      for (int i : trace_on_face[f])
                        {
                          const double xi = shape_trace(f, qf, i, b);
                          for (int j : cell_on_face[f])
                            {
                              Vec    fj, Ej;
                              double cj, dummy;
                              shape_face(f, qf, j, b, fj, cj);
                              shape_face(f, qf, j, 0, Ej, dummy);
                              if (b == 0)
                                {
                                  const Vec eps_E = scale(fj, eps);
                                  w.tc[i * Nc + j] -=
                                    (dot(eps_E, normal, dim) + tauf[0][qf] * cj) *
                                    xi * JxW;
                                }
                              else
                                {
                                  const Vec    mu_E = scale(Ej, mu);
                                  const Vec    D_f  = scale(scale(fj, mu), U_Tf);
                                  const double sgn  = (b == 1) ? 1. : -1.;
                                  const double c0q  = c0f[b][qf];
                                  const double tr0q = trc0[b][qf];
                                  double       cE_flux;
                                  const bool   cellside =
                                    (P.flux == USE_CELL) ||
                                    (P.flux == QIU_SHI && E0n > 0);
                                  if (cellside)
                                    cE_flux = sgn * (cj * dot(mu_E0, normal, dim) +
                                                     c0q * dot(mu_E, normal, dim));
                                  else
                                    cE_flux = sgn * tr0q * dot(mu_E, normal, dim);
                                  w.tc[i * Nc + j] -=
                                    (cE_flux - dot(D_f, normal, dim) -
                                     tauf[b][qf] * cj) *
                                    xi * JxW;
                                }
                            }
                        }
                    }
                  // add_tc_matrix_terms_to_tt_rhs (T:1311-1447)
                  for (int qf = 0; qf < nqf; ++qf)
                    {
                      const double JxW = G.fJxW[f * nqf + qf];
                      const double E0n = dot(d0f[0][qf], normal, dim);
                      double       term;
                      if (b == 0)
                        {
                          const Vec eps_E0f = scale(d0f[0][qf], eps);
                          term = -dot(eps_E0f, normal, dim) - tauf[0][qf] * c0f[0][qf];
                        }
                      else
                        {
                          const double mu = (b == 1) ? mun : mup;
                          const double mu_E0n =
                            dot(scale(d0f[0][qf], mu), normal, dim);
                          const Vec    D_f0 = scale(scale(d0f[b][qf], mu), U_Tf);
                          const bool   cellside =
                            (P.flux == USE_CELL) || (P.flux == QIU_SHI && E0n > 0);
                          const double c0star = cellside ? c0f[b][qf] : trc0[b][qf];
                          const double sgn    = (b == 1) ? -1. : 1.;
                          term = sgn * c0star * mu_E0n + dot(D_f0, normal, dim) +
                                 tauf[b][qf] * c0f[b][qf];
                        }
                      for (int i : trace_on_face[f])
                        w.tt_rhs[i] += term * shape_trace(f, qf, i, b) * JxW;
                    }
                  // assemble_tt_matrix (T:1451-1547)
                  const double sign = (b == 0) ? -1. : 1.;
                  for (int qf = 0; qf < nqf; ++qf)
                    {
                      const double JxW = G.fJxW[f * nqf + qf];
                      const double E0n = dot(d0f[0][qf], normal, dim);
                      for (int i : trace_on_face[f])
                        for (int j : trace_on_face[f])
                          {
                            const double xi = shape_trace(f, qf, i, b);
                            const double tr = shape_trace(f, qf, j, b);
                            if (b != 0 && (P.flux == USE_TRACE ||
                                           (P.flux == QIU_SHI && E0n <= 0)))
                              {
                                const double mu  = (b == 1) ? mun : mup;
                                const double sgn = (b == 1) ? 1. : -1.;
                                w.tt[i * Nt + j] +=
                                  sgn * dot(scale(d0f[0][qf], mu), normal, dim) *
                                  tr * xi * JxW;
                              }
                            w.tt[i * Nt + j] += sign * tauf[b][qf] * tr * xi * JxW;
                          }
                    }
                  // add_tt_matrix_terms_to_tt_rhs (T:1551-1588)
                  for (int qf = 0; qf < nqf; ++qf)
                    {
                      const double JxW = G.fJxW[f * nqf + qf];
                      for (int i : trace_on_face[f])
                        w.tt_rhs[i] += -sign * tauf[b][qf] * trc0[b][qf] *
                                       shape_trace(f, qf, i, b) * JxW;
                    }
                  // apply_nbc_on_face (T:1695-1734)
                  if (bc == 2)
                    for (int qf = 0; qf < nqf; ++qf)
                      {
                        const double JxW = G.fJxW[f * nqf + qf];
                        const double g =
                          thermo ? 0. : P.face_bc_val[(F * 3 + b) * nqf + qf];
                        for (int i : trace_on_face[f])
                          w.tt_rhs[i] += shape_trace(f, qf, i, b) * g * JxW;
                      }
                }
            }

          // ---- add_border_products_to_cc_matrix (T:1737-1923)
          for (int qf = 0; qf < nqf; ++qf)
            {
              const double JxW    = G.fJxW[f * nqf + qf];
              const double E0n    = dot(d0f[0][qf], normal, dim);
              const Vec    mun_E0 = scale(d0f[0][qf], mun);
              const Vec    mup_E0 = scale(d0f[0][qf], mup);
              const bool   cellside =
                (P.flux == USE_CELL) || (P.flux == QIU_SHI && E0n > 0);
              for (int i : cell_on_face[f])
                {
                  Vec    tq;
                  double z1, z2, z3;
                  shape_face(f, qf, i, 0, tq, z1);
                  shape_face(f, qf, i, 1, tq, z2);
                  shape_face(f, qf, i, 2, tq, z3);
                  for (int j : cell_on_face[f])
                    {
                      Vec    E, Wn, Wp;
                      double V, n, p;
                      shape_face(f, qf, j, 0, E, V);
                      shape_face(f, qf, j, 1, Wn, n);
                      shape_face(f, qf, j, 2, Wp, p);
                      double s = 0.;
                      if (Ven)
                        {
                          const Vec eps_E = scale(E, eps);
                          s += (dot(eps_E, normal, dim) * z1 +
                                tauf[0][qf] * V * z1) *
                               JxW;
                        }
                      if (nen)
                        {
                          const Vec mu_E = scale(E, mun);
                          const Vec DWn  = scale(scale(Wn, mun), U_Tf);
                          double    cE_flux;
                          if (cellside)
                            cE_flux = n * dot(mun_E0, normal, dim) +
                                      dot(mu_E, normal, dim) * c0f[1][qf];
                          else
                            cE_flux = dot(mu_E, normal, dim) * trc0[1][qf];
                          s += (cE_flux * z2 - dot(DWn, normal, dim) * z2 -
                                tauf[1][qf] * n * z2) *
                               JxW;
                        }
                      if (pen)
                        {
                          const Vec mu_E = scale(E, mup);
                          const Vec DWp  = scale(scale(Wp, mup), U_Tf);
                          double    cE_flux;
                          if (cellside)
                            cE_flux = -(p * dot(mup_E0, normal, dim) +
                                        dot(mu_E, normal, dim) * c0f[2][qf]);
                          else
                            cE_flux = -dot(mu_E, normal, dim) * trc0[2][qf];
                          s += (cE_flux * z3 - dot(DWp, normal, dim) * z3 -
                                tauf[2][qf] * p * z3) *
                               JxW;
                        }
                      w.cc[i * Nc + j] += s;
                    }
                }
            }

          // ---- add_border_products_to_cc_rhs (T:1927-2118)
          for (int qf = 0; qf < nqf; ++qf)
            {
              const double JxW = G.fJxW[f * nqf + qf];
              const double E0n = dot(d0f[0][qf], normal, dim);
              const bool   cellside =
                (P.flux == USE_CELL) || (P.flux == QIU_SHI && E0n > 0);
              double epsE0n = 0., Jn_flux = 0., Jp_flux = 0.;
              if (Ven)
                epsE0n = dot(scale(d0f[0][qf], eps), normal, dim);
              if (nen)
                {
                  const double muE0n = dot(scale(d0f[0][qf], mun), normal, dim);
                  const double DWn0n =
                    dot(scale(scale(d0f[1][qf], mun), U_Tf), normal, dim);
                  const double nn = cellside ? c0f[1][qf] : trc0[1][qf];
                  Jn_flux         = nn * muE0n - DWn0n;
                }
              if (pen)
                {
                  const double muE0n = dot(scale(d0f[0][qf], mup), normal, dim);
                  const double DWp0n =
                    dot(scale(scale(d0f[2][qf], mup), U_Tf), normal, dim);
                  const double pp = cellside ? c0f[2][qf] : trc0[2][qf];
                  Jp_flux         = -pp * muE0n - DWp0n;
                }
              for (int ii : cell_on_face[f])
                {
                  Vec    tq;
                  double z1, z2, z3;
                  shape_face(f, qf, ii, 0, tq, z1);
                  shape_face(f, qf, ii, 1, tq, z2);
                  shape_face(f, qf, ii, 2, tq, z3);
                  double s = 0.;
                  if (Ven)
                    s += (-epsE0n * z1 - tauf[0][qf] * c0f[0][qf] * z1) * JxW;
                  if (nen)
                    s += (-Jn_flux * z2 + tauf[1][qf] * c0f[1][qf] * z2) * JxW;
                  if (pen)
                    s += (-Jp_flux * z3 + tauf[2][qf] * c0f[2][qf] * z3) * JxW;
                  w.cc_rhs[ii] += s;
                }
            }

          // ---- add_trace_terms_to_cc_rhs (T:2122-2160)
          if (reconstruct)
            for (int qf = 0; qf < nqf; ++qf)
              {
                const double JxW = G.fJxW[f * nqf + qf];
                for (int b = 0; b < 3; ++b)
                  {
                    if (!P.enabled[b])
                      continue;
                    const double sign = (b == 0) ? 1. : -1.;
                    for (int i : cell_on_face[f])
                      {
                        Vec    fv;
                        double cv;
                        shape_face(f, qf, i, b, fv, cv);
                        w.cc_rhs[i] += (-dot(fv, normal, dim) +
                                        sign * tauf[b][qf] * cv) *
                                       dtr[b][qf] * JxW;
                      }
                  }
              }
        }

      // ---- LocalCondenser::condense_ct_matrix (src/local_condenser.cpp:142-160)
      if (!reconstruct && has_bc)
        for (int i = 0; i < Nc; ++i)
          for (size_t j = 0; j < cons_dof.size(); ++j)
            {
              const int    jj = cons_dof[j];
              const double mv = w.ct[i * Nt + jj];
              w.ct[i * Nt + jj] = 0.;
              w.cc_rhs[i] -= mv * cons_val[j];
            }

      if (out.dbc_local)
        {
          for (int j = 0; j < Nt; ++j)
            {
              out.dbc_local[j] = 0;
              out.dbc_value[j] = 0.;
            }
          for (size_t j = 0; j < cons_dof.size(); ++j)
            {
              out.dbc_local[cons_dof[j]] = 1;
              out.dbc_value[cons_dof[j]] = cons_val[j];
            }
        }

      if (!schur)
        {
          if (out.cc)
            std::copy(w.cc.begin(), w.cc.end(), out.cc);
          if (out.cc_rhs)
            std::copy(w.cc_rhs.begin(), w.cc_rhs.end(), out.cc_rhs);
          if (!reconstruct)
            {
              if (out.ct)
                std::copy(w.ct.begin(), w.ct.end(), out.ct);
              if (out.tc)
                std::copy(w.tc.begin(), w.tc.end(), out.tc);
              if (out.tt)
                std::copy(w.tt.begin(), w.tt.end(), out.tt);
              if (out.tt_rhs)
                std::copy(w.tt_rhs.begin(), w.tt_rhs.end(), out.tt_rhs);
            }
          return;
        }

      // ---- gauss_jordan + Schur complement (T:2651-2697)
      invert(w.cc, Nc);
      if (!reconstruct)
        {
          w.tmp.assign(Nt * Nc, 0.);
          for (int i = 0; i < Nt; ++i)
            for (int l = 0; l < Nc; ++l)
              {
                const double a = w.tc[i * Nc + l];
                if (a == 0.)
                  continue;
                for (int j = 0; j < Nc; ++j)
                  w.tmp[i * Nc + j] += a * w.cc[l * Nc + j];
              }
          for (int i = 0; i < Nt; ++i)
            {
              double s = 0.;
              for (int j = 0; j < Nc; ++j)
                s += w.tmp[i * Nc + j] * w.cc_rhs[j];
              w.tt_rhs[i] += s;
            }
          for (int i = 0; i < Nt; ++i)
            for (int l = 0; l < Nc; ++l)
              {
                const double a = w.tmp[i * Nc + l];
                if (a == 0.)
                  continue;
                for (int j = 0; j < Nt; ++j)
                  w.tt[i * Nt + j] += a * w.ct[l * Nt + j];
              }
          if (out.tt)
            std::copy(w.tt.begin(), w.tt.end(), out.tt);
          if (out.tt_rhs)
            std::copy(w.tt_rhs.begin(), w.tt_rhs.end(), out.tt_rhs);
        }
      else
        {
          for (int i = 0; i < Nc_all; ++i)
            out.update_cell[i] = 0.;
          for (int i = 0; i < Nc; ++i)
            {
              double s = 0.;
              for (int j = 0; j < Nc; ++j)
                s += w.cc[i * Nc + j] * w.cc_rhs[j];
              out.update_cell[enabled_dofs[i]] = s;
            }
        }
    }
  };
} // namespace

extern "C"
{
  int
  oracle_sizes(const OrProblem *P, int *out)
  {
    Oracle o(*P);
    out[0] = o.Nc_all;
    out[1] = o.Nc;
    out[2] = o.Nt;
    out[3] = (int)o.G.ncells;
    out[4] = (int)o.G.nfaces;
    out[5] = o.G.nqc;
    out[6] = o.G.nqf;
    out[7] = o.nb;
    out[8] = o.nf;
    return 0;
  }

  // Geometry tables for the Python side (cell/face qp reference coordinates
  // and weights, basis values).  Arrays sized by oracle_sizes.
  int
  oracle_tables(const OrProblem *P, double *cqref, double *cJxW, double *fqref,
                double *fJxW, double *cphi, double *fxi, double *fphi,
                double *cgrad)
  {
    Oracle o(*P);
    const auto &G = o.G;
    for (int q = 0; q < G.nqc; ++q)
      {
        for (int a = 0; a < 3; ++a)
          cqref[q * 3 + a] = G.cqref[q].v[a];
        cJxW[q] = G.cJxW[q];
      }
    for (int f = 0; f < G.nfaces_cell; ++f)
      for (int q = 0; q < G.nqf; ++q)
        {
          for (int a = 0; a < 3; ++a)
            fqref[(f * G.nqf + q) * 3 + a] = G.fqref[f * G.nqf + q].v[a];
          fJxW[f * G.nqf + q] = G.fJxW[f * G.nqf + q];
        }
    std::copy(G.cphi.begin(), G.cphi.end(), cphi);
    std::copy(G.fxi.begin(), G.fxi.end(), fxi);
    std::copy(G.fphi.begin(), G.fphi.end(), fphi);
    for (int q = 0; q < G.nqc; ++q)
      for (int a = 0; a < G.nb; ++a)
        for (int s = 0; s < 3; ++s)
          cgrad[(q * G.nb + a) * 3 + s] = G.cgrad[q * G.nb + a].v[s];
    return 0;
  }

  // get_local_cell_system equivalent (src/np_solver.cpp:2337-2445): the local
  // matrices of one cell before the Schur complement.
  int
  oracle_local_cell_system(const OrProblem *P, const double *cell_state,
                           const double *trace_state, long cell, int thermo,
                           double *cc, double *ct, double *tc, double *tt,
                           double *cc_rhs, double *tt_rhs)
  {
    Oracle    o(*P);
    Workspace w;
    Outputs   out{};
    out.cc     = cc;
    out.ct     = ct;
    out.tc     = tc;
    out.tt     = tt;
    out.cc_rhs = cc_rhs;
    out.tt_rhs = tt_rhs;
    o.cell_system(cell, cell_state, trace_state, nullptr, false, thermo != 0,
                  false, w, out);
    return 0;
  }

  // The local systems of every cell before the Schur complement (OpenMP).
  // With update_trace != null the reconstruction-pass cc and cc_rhs are
  // returned (ct, tc, tt, tt_rhs untouched).
  int
  oracle_local_cell_systems(const OrProblem *P, const double *cell_state,
                            const double *trace_state, const double *update_trace,
                            int thermo, double *cc, double *ct, double *tc,
                            double *tt, double *cc_rhs, double *tt_rhs, int nthreads)
  {
    Oracle     o(*P);
    const long ncells = o.G.ncells;
    const long Nc = o.Nc, Nt = o.Nt;
#ifdef _OPENMP
    if (nthreads > 0)
      omp_set_num_threads(nthreads);
#pragma omp parallel
#endif
    {
      Workspace w;
#ifdef _OPENMP
#pragma omp for schedule(static)
#endif
      for (long c = 0; c < ncells; ++c)
        {
          Outputs out{};
          out.cc     = cc + c * Nc * Nc;
          out.ct     = ct + c * Nc * Nt;
          out.tc     = tc + c * Nt * Nc;
          out.tt     = tt + c * Nt * Nt;
          out.cc_rhs = cc_rhs + c * Nc;
          out.tt_rhs = tt_rhs + c * Nt;
          o.cell_system(c, cell_state, trace_state, update_trace,
                        update_trace != nullptr, thermo != 0, false, w, out);
        }
    }
    return 0;
  }

  // Condensation pass over all cells: per-cell Schur complement tt [ncells][Nt][Nt],
  // rhs [ncells][Nt], Dirichlet flags/values [ncells][Nt].
  int
  oracle_assemble_condense(const OrProblem *P, const double *cell_state,
                           const double *trace_state, int thermo, double *tt,
                           double *tt_rhs, int *dbc_flag, double *dbc_value,
                           int nthreads)
  {
    Oracle     o(*P);
    const long ncells = o.G.ncells;
    const int  Nt     = o.Nt;
#ifdef _OPENMP
    if (nthreads > 0)
      omp_set_num_threads(nthreads);
#pragma omp parallel
#endif
    {
      Workspace w;
#ifdef _OPENMP
#pragma omp for schedule(static)
#endif
      for (long c = 0; c < ncells; ++c)
        {
          Outputs out{};
          out.tt        = tt + c * Nt * Nt;
          out.tt_rhs    = tt_rhs + c * Nt;
          out.dbc_local = dbc_flag + c * Nt;
          out.dbc_value = dbc_value + c * Nt;
          o.cell_system(c, cell_state, trace_state, nullptr, false,
                        thermo != 0, true, w, out);
        }
    }
    return 0;
  }

  // Reconstruction pass over all cells (update_cell [ncells][Nc_all]).
  int
  oracle_reconstruct(const OrProblem *P, const double *cell_state,
                     const double *trace_state, const double *update_trace,
                     int thermo, double *update_cell, int nthreads)
  {
    Oracle     o(*P);
    const long ncells = o.G.ncells;
#ifdef _OPENMP
    if (nthreads > 0)
      omp_set_num_threads(nthreads);
#pragma omp parallel
#endif
    {
      Workspace w;
#ifdef _OPENMP
#pragma omp for schedule(static)
#endif
      for (long c = 0; c < ncells; ++c)
        {
          Outputs out{};
          out.update_cell = update_cell + c * o.Nc_all;
          o.cell_system(c, cell_state, trace_state, update_trace, true,
                        thermo != 0, true, w, out);
        }
    }
    return 0;
  }

  // Recombination known answers (src/recombination_term.cpp:433-575).
  void
  oracle_srh(double ni, double tau_n, double tau_p, double n, double p,
             double rescaling, double *r, double *drn, double *drp)
  {
    const double nis = ni / rescaling;
    const double num = n * p - nis * nis;
    const double den = tau_p * (n + nis) + tau_n * (p + nis);
    *r               = num * rescaling / den;
    *drn             = p / den - num * tau_p / (den * den);
    *drp             = n / den - num * tau_n / (den * den);
  }

  double
  oracle_srh_intrinsic(double Nc, double Nv, double Ec, double Ev, double T)
  {
    return Nc * Nv * std::exp((Ev - Ec) / (KB * T));
  }
}
