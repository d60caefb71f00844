// Host-side construction of the constant per-(dim, degree, h) tables used by
// the device kernels: tensor-product Lagrange bases on Gauss-Lobatto support
// points (FE_DGQ / FE_FaceQ of deal.II 9), QGauss(k+1) rules, and the
// operators that eliminate the flux unknowns (E, Wn, Wp) of a cell through
// its mass matrix.
//
// For one component with scalar coefficients u and flux coefficients W the
// flux rows of the local system read (include/assembling_methods.template.h:
// 461-527 with the border terms of :885-1019)
//     M W - G u + C_W lambda = b_W,
// M the (block diagonal) mass matrix, G(i=(s,c), e) = int phi_e d_s phi_c,
// C_W(i, (f,m)) = int_f xi_m n_s phi_c.  Hence W = P u - Q lambda + M^-1 b_W
// with P = M^-1 G and Q = M^-1 C_W, both constant on a uniform mesh.
#pragma once

#include <cmath>
#include <vector>

namespace ddhdg
{
  struct Tables
  {
    int dim = 0, k = 0, nb = 0, nf = 0, nqc = 0, nqf = 0, F = 0;
    double h[3] = {1., 1., 1.};
    // cell quadrature
    std::vector<double> phi_c;  // [nqc][nb]
    std::vector<double> grad_c; // [nqc][nb][dim]  physical gradients
    std::vector<double> w_c;    // [nqc] JxW
    // faces (local face f: axis f/2, side f%2)
    std::vector<double> phi_f;  // [F][nqf][nb]  cell basis on face points
    std::vector<double> w_f;    // [F][nqf]      JxW
    std::vector<double> xi;     // [nqf][nf]     trace basis
    std::vector<double> fminvw; // [nf][nqf]     (face mass)^-1 * xi * w (unit face)
    std::vector<double> minv;   // [nb][nb]      inverse cell mass matrix
    // elimination operators
    std::vector<double> P;      // [dim*nb][nb]
    std::vector<double> Q;      // [dim*nb][F*nf]
    std::vector<double> PW_c;   // [nb][nqc][dim]
    std::vector<double> PW_f;   // [nb][F][nqf]   normal component
    std::vector<double> QW_c;   // [F*nf][nqc][dim]
    std::vector<double> QW_f;   // [F*nf][F][nqf] normal component
    // channel tables of the condensation kernel (contraction index first)
    std::vector<double> TLc;  // [nqc][nb]        w_q phi_a(q)
    std::vector<double> TLg;  // [nqc*dim][nb]    w_q d_s phi_a(q)
    std::vector<double> TLf;  // [F*nqf][nb]      w_fq phi_a(fq)
    std::vector<double> RTk;  // [nqc*dim][nb]    PW_e(q, s)
    std::vector<double> RTr;  // [F*nqf][nb]      PWf_e(fq)
    std::vector<double> RQk;  // [nqc*dim][F*nf]  QW_t(q, s)
    std::vector<double> RQr;  // [F*nqf][F*nf]    QWf_t(fq)
    std::vector<double> qref_c; // [nqc][3] reference coordinates
    std::vector<double> qref_f; // [F][nqf][3]
    std::vector<double> gl;     // [k+1] support points
  };

  inline double
  legendre_p(int n, double x, double *dp)
  {
    double p0 = 1., p1 = x, d0 = 0., d1 = 1.;
    if (n == 0)
      {
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
    *dp = d1;
    return p1;
  }

  // QGauss<1>(m) on [0,1], ascending.
  inline void
  gauss(int m, std::vector<double> &x, std::vector<double> &w)
  {
    x.assign(m, 0.);
    w.assign(m, 0.);
    for (int i = 0; i < m; ++i)
      {
        double t = std::cos(M_PI * (i + 0.75) / (m + 0.5));
        double d = 0.;
        for (int it = 0; it < 100; ++it)
          {
            const double p   = legendre_p(m, t, &d);
            const double del = p / d;
            t -= del;
            if (std::fabs(del) < 1e-16)
              break;
          }
        legendre_p(m, t, &d);
        x[m - 1 - i] = 0.5 * (1. + t);
        w[m - 1 - i] = 1. / ((1. - t * t) * d * d);
      }
  }

  // Gauss-Lobatto support points of degree k on [0,1] (midpoint for k = 0).
  inline std::vector<double>
  lobatto(int k)
  {
    std::vector<double> x(k + 1, 0.5);
    if (k == 0)
      return x;
    x[0] = 0.;
    x[k] = 1.;
    for (int i = 1; i < k; ++i)
      {
        double t = -std::cos(M_PI * i / k);
        for (int it = 0; it < 200; ++it)
          {
            double       d;
            const double p   = legendre_p(k, t, &d);
            const double dd  = (2. * t * d - k * (k + 1.) * p) / (1. - t * t);
            const double del = d / dd;
            t -= del;
            if (std::fabs(del) < 1e-16)
              break;
          }
        x[i] = 0.5 * (1. + t);
      }
    for (int i = 0; i <= k; ++i)
      for (int j = i + 1; j <= k; ++j)
        if (x[j] < x[i])
          std::swap(x[i], x[j]);
    return x;
  }

  inline double
  lag(const std::vector<double> &nd, int a, double x)
  {
    double r = 1.;
    for (int b = 0; b < (int)nd.size(); ++b)
      if (b != a)
        r *= (x - nd[b]) / (nd[a] - nd[b]);
    return r;
  }

  inline double
  lag_d(const std::vector<double> &nd, int a, double x)
  {
    double s = 0.;
    for (int m = 0; m < (int)nd.size(); ++m)
      {
        if (m == a)
          continue;
        double r = 1. / (nd[a] - nd[m]);
        for (int b = 0; b < (int)nd.size(); ++b)
          if (b != a && b != m)
            r *= (x - nd[b]) / (nd[a] - nd[b]);
        s += r;
      }
    return s;
  }

  // Dense inverse by Gauss-Jordan with partial pivoting (small SPD mass
  // matrices only).
  inline void
  small_inverse(std::vector<double> &A, int n)
  {
    std::vector<double> I(n * n, 0.);
    for (int i = 0; i < n; ++i)
      I[i * n + i] = 1.;
    for (int j = 0; j < n; ++j)
      {
        int p = j;
        for (int i = j + 1; i < n; ++i)
          if (std::fabs(A[i * n + j]) > std::fabs(A[p * n + j]))
            p = i;
        for (int c = 0; c < n; ++c)
          {
            std::swap(A[j * n + c], A[p * n + c]);
            std::swap(I[j * n + c], I[p * n + c]);
          }
        const double d = A[j * n + j];
        for (int c = 0; c < n; ++c)
          {
            A[j * n + c] /= d;
            I[j * n + c] /= d;
          }
        for (int i = 0; i < n; ++i)
          if (i != j)
            {
              const double f = A[i * n + j];
              if (f == 0.)
                continue;
              for (int c = 0; c < n; ++c)
                {
                  A[i * n + c] -= f * A[j * n + c];
                  I[i * n + c] -= f * I[j * n + c];
                }
            }
      }
    A = I;
  }

  inline Tables
  build_tables(int dim, int k, const double *h)
  {
    Tables T;
    T.dim = dim;
    T.k   = k;
    T.nb  = 1;
    T.nf  = 1;
    for (int i = 0; i < dim; ++i)
      T.nb *= (k + 1);
    for (int i = 0; i < dim - 1; ++i)
      T.nf *= (k + 1);
    T.nqc = T.nb;
    T.nqf = T.nf;
    T.F   = 2 * dim;
    for (int a = 0; a < 3; ++a)
      T.h[a] = (a < dim) ? h[a] : 1.;
    const int nb = T.nb, nf = T.nf, nqc = T.nqc, nqf = T.nqf, F = T.F, D = dim;

    std::vector<double> g, w;
    gauss(k + 1, g, w);
    T.gl = lobatto(k);
    const std::vector<double> &nd = T.gl;

    auto digits = [&](int idx, int nd_, int *out) {
      for (int a = 0; a < nd_; ++a)
        {
          out[a] = idx % (k + 1);
          idx /= (k + 1);
        }
    };

    double vol = 1.;
    for (int a = 0; a < D; ++a)
      vol *= T.h[a];

    T.phi_c.assign(nqc * nb, 0.);
    T.grad_c.assign(nqc * nb * D, 0.);
    T.w_c.assign(nqc, 0.);
    T.qref_c.assign(nqc * 3, 0.);
    for (int q = 0; q < nqc; ++q)
      {
        int qi[3] = {0, 0, 0};
        digits(q, D, qi);
        double ww = vol;
        for (int a = 0; a < D; ++a)
          {
            ww *= w[qi[a]];
            T.qref_c[q * 3 + a] = g[qi[a]];
          }
        T.w_c[q] = ww;
        for (int i = 0; i < nb; ++i)
          {
            int ai[3] = {0, 0, 0};
            digits(i, D, ai);
            double v = 1.;
            for (int a = 0; a < D; ++a)
              v *= lag(nd, ai[a], g[qi[a]]);
            T.phi_c[q * nb + i] = v;
            for (int s = 0; s < D; ++s)
              {
                double gg = 1.;
                for (int a = 0; a < D; ++a)
                  gg *= (a == s) ? lag_d(nd, ai[a], g[qi[a]]) / T.h[a] :
                                   lag(nd, ai[a], g[qi[a]]);
                T.grad_c[(q * nb + i) * D + s] = gg;
              }
          }
      }

    T.phi_f.assign(F * nqf * nb, 0.);
    T.w_f.assign(F * nqf, 0.);
    T.xi.assign(nqf * nf, 0.);
    T.qref_f.assign(F * nqf * 3, 0.);
    std::vector<double> wunit(nqf, 1.);
    for (int qf = 0; qf < nqf; ++qf)
      {
        int qi[2] = {0, 0};
        digits(qf, D - 1, qi);
        for (int t = 0; t < D - 1; ++t)
          wunit[qf] *= w[qi[t]];
        for (int m = 0; m < nf; ++m)
          {
            int mi[2] = {0, 0};
            digits(m, D - 1, mi);
            double v = 1.;
            for (int t = 0; t < D - 1; ++t)
              v *= lag(nd, mi[t], g[qi[t]]);
            T.xi[qf * nf + m] = v;
          }
      }
    for (int f = 0; f < F; ++f)
      {
        const int a    = f / 2;
        const int side = f % 2;
        double    area = 1.;
        for (int b = 0; b < D; ++b)
          if (b != a)
            area *= T.h[b];
        for (int qf = 0; qf < nqf; ++qf)
          {
            int qi[2] = {0, 0};
            digits(qf, D - 1, qi);
            double xr[3] = {0., 0., 0.};
            xr[a]        = side ? 1. : 0.;
            for (int t = 0; t < D - 1; ++t)
              xr[(a + 1 + t) % D] = g[qi[t]];
            for (int c = 0; c < 3; ++c)
              T.qref_f[(f * nqf + qf) * 3 + c] = xr[c];
            T.w_f[f * nqf + qf] = area * wunit[qf];
            for (int i = 0; i < nb; ++i)
              {
                int ai[3] = {0, 0, 0};
                digits(i, D, ai);
                double v = 1.;
                for (int b = 0; b < D; ++b)
                  v *= lag(nd, ai[b], xr[b]);
                T.phi_f[(f * nqf + qf) * nb + i] = v;
              }
          }
      }

    // face mass matrix on the unit face and (Mf^-1 xi w)
    {
      std::vector<double> Mf(nf * nf, 0.);
      for (int qf = 0; qf < nqf; ++qf)
        for (int i = 0; i < nf; ++i)
          for (int j = 0; j < nf; ++j)
            Mf[i * nf + j] += T.xi[qf * nf + i] * T.xi[qf * nf + j] * wunit[qf];
      small_inverse(Mf, nf);
      T.fminvw.assign(nf * nqf, 0.);
      for (int m = 0; m < nf; ++m)
        for (int qf = 0; qf < nqf; ++qf)
          {
            double s = 0.;
            for (int j = 0; j < nf; ++j)
              s += Mf[m * nf + j] * T.xi[qf * nf + j];
            T.fminvw[m * nqf + qf] = s * wunit[qf];
          }
    }

    // cell mass matrix and its inverse
    std::vector<double> M(nb * nb, 0.);
    for (int q = 0; q < nqc; ++q)
      for (int i = 0; i < nb; ++i)
        for (int j = 0; j < nb; ++j)
          M[i * nb + j] += T.phi_c[q * nb + i] * T.phi_c[q * nb + j] * T.w_c[q];
    small_inverse(M, nb);
    T.minv = M;

    // G((s,c), e) and C_W((s,c),(f,m))
    std::vector<double> G(D * nb * nb, 0.), CW(D * nb * F * nf, 0.);
    for (int s = 0; s < D; ++s)
      for (int c = 0; c < nb; ++c)
        for (int e = 0; e < nb; ++e)
          {
            double acc = 0.;
            for (int q = 0; q < nqc; ++q)
              acc += T.phi_c[q * nb + e] * T.grad_c[(q * nb + c) * D + s] * T.w_c[q];
            G[(s * nb + c) * nb + e] = acc;
          }
    for (int f = 0; f < F; ++f)
      {
        const int    a  = f / 2;
        const double ns = (f % 2) ? 1. : -1.;
        for (int c = 0; c < nb; ++c)
          for (int m = 0; m < nf; ++m)
            {
              double acc = 0.;
              for (int qf = 0; qf < nqf; ++qf)
                acc += T.xi[qf * nf + m] * T.phi_f[(f * nqf + qf) * nb + c] *
                       T.w_f[f * nqf + qf];
              CW[(a * nb + c) * (F * nf) + f * nf + m] = ns * acc;
            }
      }
    T.P.assign(D * nb * nb, 0.);
    T.Q.assign(D * nb * F * nf, 0.);
    for (int s = 0; s < D; ++s)
      for (int c = 0; c < nb; ++c)
        {
          for (int e = 0; e < nb; ++e)
            {
              double acc = 0.;
              for (int cc = 0; cc < nb; ++cc)
                acc += T.minv[c * nb + cc] * G[(s * nb + cc) * nb + e];
              T.P[(s * nb + c) * nb + e] = acc;
            }
          for (int t = 0; t < F * nf; ++t)
            {
              double acc = 0.;
              for (int cc = 0; cc < nb; ++cc)
                acc += T.minv[c * nb + cc] * CW[(s * nb + cc) * (F * nf) + t];
              T.Q[(s * nb + c) * (F * nf) + t] = acc;
            }
        }

    T.PW_c.assign(nb * nqc * D, 0.);
    T.PW_f.assign(nb * F * nqf, 0.);
    T.QW_c.assign(F * nf * nqc * D, 0.);
    T.QW_f.assign(F * nf * F * nqf, 0.);
    for (int e = 0; e < nb; ++e)
      {
        for (int q = 0; q < nqc; ++q)
          for (int s = 0; s < D; ++s)
            {
              double acc = 0.;
              for (int c = 0; c < nb; ++c)
                acc += T.P[(s * nb + c) * nb + e] * T.phi_c[q * nb + c];
              T.PW_c[(e * nqc + q) * D + s] = acc;
            }
        for (int f = 0; f < F; ++f)
          {
            const int    a  = f / 2;
            const double ns = (f % 2) ? 1. : -1.;
            for (int qf = 0; qf < nqf; ++qf)
              {
                double acc = 0.;
                for (int c = 0; c < nb; ++c)
                  acc += T.P[(a * nb + c) * nb + e] * T.phi_f[(f * nqf + qf) * nb + c];
                T.PW_f[(e * F + f) * nqf + qf] = ns * acc;
              }
          }
      }
    for (int t = 0; t < F * nf; ++t)
      {
        for (int q = 0; q < nqc; ++q)
          for (int s = 0; s < D; ++s)
            {
              double acc = 0.;
              for (int c = 0; c < nb; ++c)
                acc += T.Q[(s * nb + c) * (F * nf) + t] * T.phi_c[q * nb + c];
              T.QW_c[(t * nqc + q) * D + s] = acc;
            }
        for (int f = 0; f < F; ++f)
          {
            const int    a  = f / 2;
            const double ns = (f % 2) ? 1. : -1.;
            for (int qf = 0; qf < nqf; ++qf)
              {
                double acc = 0.;
                for (int c = 0; c < nb; ++c)
                  acc += T.Q[(a * nb + c) * (F * nf) + t] *
                         T.phi_f[(f * nqf + qf) * nb + c];
                T.QW_f[(t * F + f) * nqf + qf] = ns * acc;
              }
          }
      }
    const int Fq = F * nqf, Ft = F * nf;
    T.TLc.assign(nqc * nb, 0.);
    T.TLg.assign(nqc * D * nb, 0.);
    T.TLf.assign(Fq * nb, 0.);
    T.RTk.assign(nqc * D * nb, 0.);
    T.RTr.assign(Fq * nb, 0.);
    T.RQk.assign(nqc * D * Ft, 0.);
    T.RQr.assign(Fq * Ft, 0.);
    for (int q = 0; q < nqc; ++q)
      for (int a = 0; a < nb; ++a)
        {
          T.TLc[q * nb + a] = T.w_c[q] * T.phi_c[q * nb + a];
          for (int s = 0; s < D; ++s)
            {
              T.TLg[(q * D + s) * nb + a] = T.w_c[q] * T.grad_c[(q * nb + a) * D + s];
              T.RTk[(q * D + s) * nb + a] = T.PW_c[(a * nqc + q) * D + s];
            }
        }
    for (int q = 0; q < nqc; ++q)
      for (int s = 0; s < D; ++s)
        for (int t = 0; t < Ft; ++t)
          T.RQk[(q * D + s) * Ft + t] = T.QW_c[(t * nqc + q) * D + s];
    for (int f = 0; f < F; ++f)
      for (int qf = 0; qf < nqf; ++qf)
        {
          const int fq = f * nqf + qf;
          for (int a = 0; a < nb; ++a)
            {
              T.TLf[fq * nb + a] = T.w_f[fq] * T.phi_f[fq * nb + a];
              T.RTr[fq * nb + a] = T.PW_f[(a * F + f) * nqf + qf];
            }
          for (int t = 0; t < Ft; ++t)
            T.RQr[fq * Ft + t] = T.QW_f[(t * F + f) * nqf + qf];
        }
    return T;
  }
} // namespace ddhdg
