// The reference's per-cell algorithm as written, on the GPU (sm_100a, FP64).
//
// For every cell the full local HDG system of the enabled components,
//     cc [Nc][Nc], ct [Nc][Nt], tc [Nt][Nc], tt [Nt][Nt], cc_rhs [Nc], tt_rhs [Nt]
// (Nc = enabled cell dofs, fluxes included; Nt = restricted trace dofs), is
// assembled term by term like include/assembling_methods.template.h:134-2160
// (volume products :269-760, ct :885-1141, tc :1145-1447, tt :1451-1588,
// Dirichlet projection :1592-1691, Neumann :1695-1734, border products
// :1737-2118, trace terms of the reconstruction :2122-2160), the Dirichlet
// columns of ct are folded into cc_rhs (src/local_condenser.cpp:142-160), and
// the Schur complement tt + tc cc^-1 [ct | cc_rhs] (:2651-2686) follows from
// an LU factorisation of the row-equilibrated cc with partial pivoting.  The
// reconstruction pass assembles cc and cc_rhs again with the trace update
// and solves (:2688-2697), as the reference does.
//
// This is the plain FP64 GPU path the block-eliminated kernels
// (hdg_condense3.cuh, hdg_condense.cuh) are measured against, and, stopped
// before the Schur step, the per-cell probe ddhdg_local_cell_system
// (get_local_cell_system, src/np_solver.cpp:2337-2445).
//
// One CTA of PlainTPB threads per cell (persistent grid).  The workspace of a
// cell (coefficients, point data, the augmented matrix [cc | cc_rhs | ct],
// tt, tt_rhs) lives in shared memory when it fits (2D k <= 2, 3D k = 1), in
// a per-CTA slice of a global buffer otherwise; tc always lives in a per-CTA
// global slice (written once and read once per cell, it stays in L2).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "hdg_kernels.cuh"

namespace ddhdg
{
  constexpr int PlainTPB = 256;

  enum PlainMode
  {
    PlainCondense    = 0, // tt, rhs, dflag, dval (like ddhdg_assemble_condense)
    PlainProbe       = 1, // the unreduced local system of listed cells
    PlainReconstruct = 2  // update_cell from a trace update
  };

  struct PlainArgs
  {
    int            mode;
    int64_t        nlist;      // probe: number of listed cells
    const int64_t *cells;      // probe: the listed cells (device)
    double *cc, *ct, *tc, *tt, *c, *t; // probe outputs [nlist][...] (any may be null)
    const double *update_trace; // reconstruct: full trace update [nfaces][3][nf]
    double       *update_cell;  // reconstruct: [ncells][Nc_all]
    double       *wscratch;     // per-CTA workspace slices, or null (shared memory)
    double       *tcscratch;    // per-CTA tc slices [Nt][Nc]
    int64_t       wstride;      // doubles per CTA slice of wscratch
  };

  struct PlainOff
  {
    int coef, lam, dlam, c0, W0, qc, c0f, W0n, tr0, dtr, tau, bcs, dfl, dvl, rs, A, TT, TR, total;
    int Nc, Nt, ldA;
  };

  __host__ __device__ inline PlainOff
  plain_layout(int dim, int nb, int nf, int ncomp, int mode)
  {
    const int F = 2 * dim, Fq = F * nf;
    PlainOff  o;
    o.Nc      = ncomp * (dim + 1) * nb;
    o.Nt      = F * ncomp * nf;
    // [cc | cc_rhs | ct] with an odd leading dimension (no bank conflicts
    // down a column)
    o.ldA = (mode == PlainReconstruct) ? o.Nc + 1 : o.Nc + 1 + o.Nt;
    o.ldA |= 1;
    int  p    = 0;
    auto take = [&p](int n) {
      const int r = p;
      p += (n + 1) & ~1;
      return r;
    };
    o.coef  = take(3 * (dim + 1) * nb);
    o.lam   = take(F * 3 * nf);
    o.dlam  = take(F * 3 * nf);
    o.c0    = take(3 * nb);
    o.W0    = take(3 * dim * nb);
    o.qc    = take(6 * nb);
    o.c0f   = take(3 * Fq);
    o.W0n   = take(3 * Fq);
    o.tr0   = take(3 * Fq);
    o.dtr   = take(3 * Fq);
    o.tau   = take(F * 3);
    o.bcs   = take(F * 3);
    o.dfl   = take(o.Nt);
    o.dvl   = take(o.Nt);
    o.rs    = take(o.Nc);
    o.A     = take(o.Nc * o.ldA);
    o.TT    = take(o.Nt * o.Nt);
    o.TR    = take(o.Nt);
    o.total = p;
    return o;
  }

  // The plain kernel.  WS_GLOBAL: the workspace lives in wscratch (large
  // cells) instead of dynamic shared memory.
  template <int DIM, int K, bool WS_GLOBAL>
  __global__ void __launch_bounds__(PlainTPB)
  plain_kernel(const KParams P, const PlainArgs A_)
  {
    using Dm          = Dims<DIM, K>;
    constexpr int nb  = Dm::nb;
    constexpr int nf  = Dm::nf;
    constexpr int nqc = Dm::nqc;
    constexpr int nqf = Dm::nqf;
    constexpr int F   = Dm::F;
    constexpr int Fq  = F * nqf;
    constexpr int NCA = Dm::Nc_all;
    constexpr int T   = PlainTPB;
    extern __shared__ double smem[];
    __shared__ int    sh_piv;
    __shared__ double sh_pmax;

    const int  tid   = threadIdx.x;
    const int  ncomp = P.ncomp;
    const int  mode  = A_.mode;
    const bool recon = mode == PlainReconstruct;

    const PlainOff wo  = plain_layout(DIM, nb, nf, ncomp, mode);
    const int      Nc  = wo.Nc, Nt = wo.Nt, ldA = wo.ldA;
    const int      NR  = recon ? 1 : 1 + Nt; // right-hand-side columns
    double        *ws  = WS_GLOBAL ? A_.wscratch + (int64_t)blockIdx.x * A_.wstride : smem;
    double        *coef = ws + wo.coef, *lam = ws + wo.lam, *dlam = ws + wo.dlam, *c0 = ws + wo.c0,
           *W0 = ws + wo.W0, *qc = ws + wo.qc, *c0f = ws + wo.c0f, *W0n = ws + wo.W0n,
           *tr0 = ws + wo.tr0, *dtr = ws + wo.dtr, *taus = ws + wo.tau, *bcs = ws + wo.bcs,
           *dfl = ws + wo.dfl, *dvl = ws + wo.dvl, *rs = ws + wo.rs, *A = ws + wo.A,
           *TT = ws + wo.TT, *TR = ws + wo.TR;
    double *TC = A_.tcscratch ? A_.tcscratch + (int64_t)blockIdx.x * Nt * Nc : nullptr;

    const double *tb     = P.tables;
    const double *phi_c  = tb + P.to.phi_c;
    const double *grad_c = tb + P.to.grad_c;
    const double *w_c    = tb + P.to.w_c;
    const double *phi_f  = tb + P.to.phi_f;
    const double *w_f    = tb + P.to.w_f;
    const double *xi     = tb + P.to.xi;

    const double eps = P.eps, mun = P.mun, mup = P.mup, U_T = P.U_T;
    const bool   thermo   = P.thermo != 0;
    const bool   phi_mode = thermo || P.phi_linearize;
    const double ds       = (P.jfix & 1) ? -1. : 1.;
    const int    flux     = P.flux;
    int          ce_of[3] = {-1, -1, -1};
    for (int c = 0; c < ncomp; ++c)
      ce_of[P.comps[c]] = c;
    const bool nen = ce_of[1] >= 0, pen = ce_of[2] >= 0;

    // node a lies on local face f (Gauss-Lobatto support: first / last
    // node along the face's axis)
    auto on_face = [](int a, int f) {
      const int ax = f / 2;
      int       d  = a;
      for (int s = 0; s < ax; ++s)
        d /= (K + 1);
      return (d % (K + 1)) == ((f & 1) ? K : 0);
    };

    const int64_t nwork = (mode == PlainProbe) ? A_.nlist : P.ncells;
    for (int64_t wi = (mode == PlainProbe ? 0 : P.cell0) + blockIdx.x; wi < nwork; wi += gridDim.x)
      {
        const int64_t cell = (mode == PlainProbe) ? A_.cells[wi] : wi;
        // ------------------------------------------------------ state
        const double *cs = P.cell_state + cell * NCA;
        for (int i = tid; i < NCA; i += T)
          coef[i] = cs[i];
        for (int i = tid; i < F * 3 * nf; i += T)
          {
            const int64_t Fi = face_index(P, cell, i / (3 * nf), DIM);
            lam[i]           = P.trace_state[Fi * 3 * nf + (i % (3 * nf))];
            dlam[i]          = recon ? A_.update_trace[Fi * 3 * nf + (i % (3 * nf))] : 0.;
          }
        for (int i = tid; i < F * 3; i += T)
          {
            const int     f  = i / 3, b = i % 3;
            const int64_t Fi = face_index(P, cell, f, DIM);
            taus[i] = P.tau_table ? P.tau_table[(cell * F + f) * 3 + b] : P.tau[b];
            bcs[i]  = (double)P.face_bc[Fi * 3 + b];
          }
        __syncthreads();

        // ------------------------ prepare_data_on_cell / face quadrature points
        for (int i = tid; i < 3 * (DIM + 1) * nqc; i += T)
          {
            const int     b  = i / ((DIM + 1) * nqc);
            const int     s  = (i / nqc) % (DIM + 1);
            const int     q  = i % nqc;
            const double *cf = coef + (b * (DIM + 1) + s) * nb;
            double        v  = 0.;
            for (int a = 0; a < nb; ++a)
              v += phi_c[q * nb + a] * cf[a];
            if (s < DIM)
              W0[(b * DIM + s) * nqc + q] = v;
            else
              c0[b * nqc + q] = v;
          }
        for (int i = tid; i < 3 * Fq; i += T)
          {
            const int     b  = i / Fq;
            const int     fq = i % Fq;
            const int     f = fq / nqf, qf = fq % nqf;
            const double  sg = (f & 1) ? 1. : -1.;
            const double *ph = phi_f + fq * nb;
            const double *cS = coef + (b * (DIM + 1) + DIM) * nb;
            const double *cW = coef + (b * (DIM + 1) + f / 2) * nb;
            double        u = 0., wn = 0., t = 0., dt = 0.;
            for (int a = 0; a < nb; ++a)
              {
                u += ph[a] * cS[a];
                wn += ph[a] * cW[a];
              }
            for (int m = 0; m < nf; ++m)
              {
                t += xi[qf * nf + m] * lam[(f * 3 + b) * nf + m];
                dt += xi[qf * nf + m] * dlam[(f * 3 + b) * nf + m];
              }
            c0f[i] = u;
            W0n[i] = sg * wn;
            tr0[i] = t;
            dtr[i] = dt;
          }
        __syncthreads();
        for (int q = tid; q < nqc; q += T)
          {
            const double V0 = c0[q], n0 = c0[nqc + q], p0 = c0[2 * nqc + q];
            double       r = 0., drn = 0., drp = 0.;
            if (nen || pen)
              {
                // src/recombination_term.cpp:433-575 (SRH), :116-160 (linear)
                const double rf_ = P.n_rescale;
                if (P.rec_type == 1)
                  {
                    const double ni  = P.srh_ni / rf_;
                    const double num = n0 * p0 - ni * ni;
                    const double den = P.srh_tau_p * (n0 + ni) + P.srh_tau_n * (p0 + ni);
                    r                = num * rf_ / den;
                    drn              = p0 / den - num * P.srh_tau_p / (den * den);
                    drp              = n0 / den - num * P.srh_tau_n / (den * den);
                  }
                else
                  {
                    const int64_t idx = cell * nqc + q;
                    const double  a_  = P.rec_a ? P.rec_a[idx] : 0.;
                    const double  b_  = P.rec_b ? P.rec_b[idx] : 0.;
                    const double  c_  = P.rec_c ? P.rec_c[idx] : 0.;
                    r                 = a_ + (b_ * n0 + c_ * p0) * rf_;
                    drn               = b_;
                    drp               = c_;
                  }
                r /= P.rec_rescale;
                drn /= P.rec_rescale;
                drp /= P.rec_rescale;
                if (P.jfix & 2)
                  {
                    drn *= rf_;
                    drp *= rf_;
                  }
              }
            double phider = 0., phirhs = 0.;
            if (phi_mode)
              {
                // Boltzmann terms of T:442-459 with the quasi Fermi
                // potentials of include/solver.h:343-376
                const double KbT = KB_ * P.T / (Q_ * P.V_rescale);
                const double evr = P.ev / (Q_ * P.V_rescale);
                const double ecr = P.ec / (Q_ * P.V_rescale);
                double       phn = 0., php = 0.;
                if (!thermo)
                  {
                    const double U  = P.T * (KB_ / Q_);
                    const double Vp = V0 * P.V_rescale;
                    if (nen)
                      phn = (Vp - P.ec / Q_ - U * log(n0 * P.n_rescale / P.nc)) / P.V_rescale;
                    if (pen)
                      php = (Vp - P.ev / Q_ + U * log(p0 * P.n_rescale / P.nv)) / P.V_rescale;
                  }
                const double e1 = exp((evr - V0 + php) / KbT);
                const double e2 = exp((V0 - phn - ecr) / KbT);
                phider          = -1. / P.n_rescale * (P.nv / KbT * e1 + P.nc / KbT * e2);
                phirhs          = 1. / P.n_rescale * (P.nv * e1 - P.nc * e2);
              }
            qc[0 * nqc + q] = r;
            qc[1 * nqc + q] = drn;
            qc[2 * nqc + q] = drp;
            qc[3 * nqc + q] = phider;
            qc[4 * nqc + q] = phirhs;
            qc[5 * nqc + q] = ce_of[0] >= 0 ? P.doping[cell * nqc + q] : 0.;
          }
        for (int i = tid; i < Nt; i += T)
          {
            dfl[i] = 0.;
            dvl[i] = 0.;
          }
        __syncthreads();

        // ---------------------------- Dirichlet L2 projection (T:1592-1691)
        if (!recon)
          for (int i = tid; i < F * ncomp; i += T)
            {
              const int f = i / ncomp, ce = i % ncomp, b = P.comps[ce];
              if (bcs[f * 3 + b] != 1.)
                continue;
              const int64_t Fi = face_index(P, cell, f, DIM);
              double        M[nf * nf], x[nf];
              for (int a = 0; a < nf * nf; ++a)
                M[a] = 0.;
              for (int a = 0; a < nf; ++a)
                x[a] = 0.;
              for (int qf = 0; qf < nqf; ++qf)
                {
                  const double w   = w_f[f * nqf + qf];
                  const double val = thermo ? 0. :
                                              P.face_bc_val[(Fi * 3 + b) * nqf + qf] -
                                                tr0[b * Fq + f * nqf + qf];
                  for (int a = 0; a < nf; ++a)
                    {
                      const double xa = xi[qf * nf + a];
                      for (int c = 0; c < nf; ++c)
                        M[a * nf + c] += xa * xi[qf * nf + c] * w;
                      x[a] += xa * val * w;
                    }
                }
              // Cholesky M = L L^T (LAPACKFullMatrix::compute_cholesky, T:1676-1678)
              for (int a = 0; a < nf; ++a)
                {
                  double d = M[a * nf + a];
                  for (int c = 0; c < a; ++c)
                    d -= M[a * nf + c] * M[a * nf + c];
                  d              = sqrt(d);
                  M[a * nf + a] = d;
                  for (int r2 = a + 1; r2 < nf; ++r2)
                    {
                      double v = M[r2 * nf + a];
                      for (int c = 0; c < a; ++c)
                        v -= M[r2 * nf + c] * M[a * nf + c];
                      M[r2 * nf + a] = v / d;
                    }
                }
              for (int a = 0; a < nf; ++a)
                {
                  double v = x[a];
                  for (int c = 0; c < a; ++c)
                    v -= M[a * nf + c] * x[c];
                  x[a] = v / M[a * nf + a];
                }
              for (int a = nf - 1; a >= 0; --a)
                {
                  double v = x[a];
                  for (int c = a + 1; c < nf; ++c)
                    v -= M[c * nf + a] * x[c];
                  x[a] = v / M[a * nf + a];
                }
              for (int a = 0; a < nf; ++a)
                {
                  const int j = (f * ncomp + ce) * nf + a;
                  dfl[j]      = 1.;
                  dvl[j]      = x[a];
                }
            }

        // ------------------------------------------------------- cc
        // entry (i, j): volume products (T:269-532) and border products of
        // every face holding both nodes (T:1737-1923)
        for (int idx = tid; idx < Nc * Nc; idx += T)
          {
            const int i = idx / Nc, j = idx % Nc;
            const int bi = P.comps[i / ((DIM + 1) * nb)], si = (i / nb) % (DIM + 1), ai = i % nb;
            const int bj = P.comps[j / ((DIM + 1) * nb)], sj = (j / nb) % (DIM + 1), aj = j % nb;
            double    s  = 0.;
            // the (test, trial) kinds with a volume term at all (the others
            // are structural zeros of the reference's loops)
            bool vol;
            if (bi == 0)
              vol = (si < DIM) ? (bj == 0 && (sj == DIM || sj == si))
                               : ((bj == 0 && sj < DIM) ||
                                  (sj == DIM && (phi_mode ? bj == 0 : bj != 0)));
            else
              vol = (si < DIM) ? (bj == bi && (sj == DIM || sj == si))
                               : (bj == bi || (bj == 0 && sj < DIM) || (sj == DIM && bj != 0));
            for (int q = 0; vol && q < nqc; ++q)
              {
                const double  w  = w_c[q];
                const double  pi = phi_c[q * nb + ai], pj = phi_c[q * nb + aj];
                const double *gi = grad_c + (q * nb + ai) * DIM;
                double        v  = 0.;
                if (bi == 0)
                  {
                    if (si < DIM)
                      {
                        if (bj == 0 && sj == DIM)
                          v = -pj * gi[si];
                        else if (bj == 0 && sj == si)
                          v = pj * pi;
                      }
                    else if (bj == 0 && sj < DIM)
                      v = -eps * pj * gi[sj];
                    else if (sj == DIM)
                      {
                        if (phi_mode)
                          v = (bj == 0) ? -qc[3 * nqc + q] * pj * pi : 0.;
                        else
                          v = (bj == 1) ? pj * pi : (bj == 2) ? -pj * pi : 0.;
                      }
                  }
                else
                  {
                    const double mu = (bi == 1) ? mun : mup;
                    if (si < DIM)
                      {
                        if (bj == bi && sj == DIM)
                          v = -pj * gi[si];
                        else if (bj == bi && sj == si)
                          v = pj * pi;
                      }
                    else
                      {
                        if (bj == bi && sj == DIM)
                          {
                            double e0g = 0.;
                            for (int d = 0; d < DIM; ++d)
                              e0g += W0[d * nqc + q] * gi[d];
                            v += ((bi == 1) ? -1. : 1.) * pj * mu * e0g;
                          }
                        if (bj == 0 && sj < DIM)
                          v += ((bi == 1) ? ds * c0[nqc + q] : -ds * c0[2 * nqc + q]) * mu * pj * gi[sj];
                        if (bj == bi && sj < DIM)
                          v += U_T * mu * pj * gi[sj];
                        if (sj == DIM && bj == 1)
                          v -= qc[1 * nqc + q] * pj * pi;
                        if (sj == DIM && bj == 2)
                          v -= qc[2 * nqc + q] * pj * pi;
                      }
                  }
                s += v * w;
              }
            // border products: the test function is a scalar, the trial a
            // scalar or the normal flux component, both on the face
            if (si == DIM)
              for (int f = 0; f < F; ++f)
                {
                  if (!on_face(ai, f) || !on_face(aj, f))
                    continue;
                  const int    ax = f / 2;
                  const double sg = (f & 1) ? 1. : -1.;
                  if (sj < DIM && sj != ax)
                    continue;
                  for (int qf = 0; qf < nqf; ++qf)
                    {
                      const int    fq  = f * nqf + qf;
                      const double w   = w_f[fq];
                      const double zi  = phi_f[fq * nb + ai], pj = phi_f[fq * nb + aj];
                      const double E0n = W0n[fq];
                      const bool   cs_ = (flux == 0) || (flux == 2 && E0n > 0.);
                      double       v   = 0.;
                      if (bi == 0)
                        {
                          if (bj == 0 && sj < DIM)
                            v = eps * sg * pj;
                          else if (bj == 0)
                            v = taus[f * 3] * pj;
                        }
                      else
                        {
                          const double mu  = (bi == 1) ? mun : mup;
                          const double sgn = (bi == 1) ? 1. : -1.;
                          const double tau = taus[f * 3 + bi];
                          if (bj == 0 && sj < DIM)
                            v = sgn * mu * sg * pj * (cs_ ? c0f[bi * Fq + fq] : tr0[bi * Fq + fq]);
                          else if (bj == bi && sj == DIM)
                            v = (cs_ ? sgn * mu * E0n : 0.) * pj - tau * pj;
                          else if (bj == bi && sj < DIM)
                            v = -U_T * mu * sg * pj;
                        }
                      s += v * zi * w;
                    }
                }
            A[i * ldA + j] = s;
          }

        // ------------------------------------------------------- cc_rhs
        // volume residual (T:536-760), -ct lambda0 (T:1023-1141), border
        // residual (T:1927-2118) and, in the reconstruction, the trace
        // update terms (T:2122-2160)
        for (int i = tid; i < Nc; i += T)
          {
            const int bi = P.comps[i / ((DIM + 1) * nb)], si = (i / nb) % (DIM + 1), ai = i % nb;
            double    s  = 0.;
            for (int q = 0; q < nqc; ++q)
              {
                const double  w  = w_c[q];
                const double  pi = phi_c[q * nb + ai];
                const double *gi = grad_c + (q * nb + ai) * DIM;
                const double  u0 = c0[bi * nqc + q];
                double        v  = 0.;
                if (si < DIM)
                  v = u0 * gi[si] - W0[(bi * DIM + si) * nqc + q] * pi;
                else if (bi == 0)
                  {
                    double e0g = 0.;
                    for (int d = 0; d < DIM; ++d)
                      e0g += W0[d * nqc + q] * gi[d];
                    v = eps * e0g + qc[5 * nqc + q] * pi;
                    v += phi_mode ? qc[4 * nqc + q] * pi : (-c0[nqc + q] + c0[2 * nqc + q]) * pi;
                  }
                else
                  {
                    const double mu = (bi == 1) ? mun : mup;
                    const double sg = (bi == 1) ? 1. : -1.;
                    double       jg = 0.;
                    for (int d = 0; d < DIM; ++d)
                      jg += (sg * u0 * mu * W0[d * nqc + q] - U_T * mu * W0[(bi * DIM + d) * nqc + q]) * gi[d];
                    v = qc[q] * pi + jg;
                  }
                s += v * w;
              }
            for (int f = 0; f < F; ++f)
              {
                if (!on_face(ai, f))
                  continue;
                const int    ax  = f / 2;
                const double sg  = (f & 1) ? 1. : -1.;
                const double tau = taus[f * 3 + bi];
                for (int qf = 0; qf < nqf; ++qf)
                  {
                    const int    fq  = f * nqf + qf;
                    const double w   = w_f[fq];
                    const double z   = phi_f[fq * nb + ai];
                    const double t0  = tr0[bi * Fq + fq];
                    const double E0n = W0n[fq];
                    double       v   = 0.;
                    if (si < DIM)
                      {
                        if (si == ax)
                          v = -t0 * sg * z - (recon ? sg * z * dtr[bi * Fq + fq] : 0.);
                      }
                    else
                      {
                        const bool cs_ = (flux == 0) || (flux == 2 && E0n > 0.);
                        if (bi == 0)
                          v = tau * t0 * z - eps * E0n * z - tau * c0f[fq] * z;
                        else
                          {
                            const double mu  = (bi == 1) ? mun : mup;
                            const double sgn = (bi == 1) ? 1. : -1.;
                            const double cst = cs_ ? c0f[bi * Fq + fq] : t0;
                            const double J   = sgn * cst * mu * E0n - U_T * mu * W0n[bi * Fq + fq];
                            v = -tau * t0 * z - J * z + tau * c0f[bi * Fq + fq] * z;
                          }
                        if (recon)
                          v += ((bi == 0) ? 1. : -1.) * tau * z * dtr[bi * Fq + fq];
                      }
                    s += v * w;
                  }
              }
            A[i * ldA + Nc] = s;
          }

        if (!recon)
          {
            // --------------------------------------------------- ct (T:885-1019)
            for (int idx = tid; idx < Nc * Nt; idx += T)
              {
                const int i = idx / Nt, j = idx % Nt;
                const int ci = i / ((DIM + 1) * nb), si = (i / nb) % (DIM + 1), ai = i % nb;
                const int f = j / (ncomp * nf), cj = (j / nf) % ncomp, m = j % nf;
                double    s = 0.;
                if (ci == cj && on_face(ai, f) && (si == DIM || si == f / 2))
                  {
                    const int    b  = P.comps[ci];
                    const double sg = (f & 1) ? 1. : -1.;
                    for (int qf = 0; qf < nqf; ++qf)
                      {
                        const int    fq  = f * nqf + qf;
                        const double w   = w_f[fq];
                        const double z   = phi_f[fq * nb + ai];
                        const double tr  = xi[qf * nf + m];
                        const double E0n = W0n[fq];
                        const bool   upw = (flux == 1) || (flux == 2 && E0n <= 0.);
                        double       v;
                        if (si < DIM)
                          v = tr * sg * z;
                        else if (b == 0)
                          v = -taus[f * 3] * tr * z;
                        else
                          {
                            const double mu  = (b == 1) ? mun : mup;
                            const double sgn = (b == 1) ? 1. : -1.;
                            v = ((upw ? sgn * mu * E0n : 0.) + taus[f * 3 + b]) * tr * z;
                          }
                        s += v * w;
                      }
                  }
                A[i * ldA + Nc + 1 + j] = s;
              }
            // ------------------------------------- tc (T:1145-1307), tt (T:1451-1547)
            for (int idx = tid; idx < Nt * Nc; idx += T)
              {
                const int i = idx / Nc, j = idx % Nc;
                const int f = i / (ncomp * nf), ci = (i / nf) % ncomp, m = i % nf;
                const int b = P.comps[ci];
                const int cj = j / ((DIM + 1) * nb), sj = (j / nb) % (DIM + 1), aj = j % nb;
                const int bj = P.comps[cj];
                double    s  = 0.;
                if (bcs[f * 3 + b] != 1. && on_face(aj, f) && (sj == DIM || sj == f / 2) &&
                    (bj == b || (bj == 0 && sj < DIM)))
                  {
                    const double sg = (f & 1) ? 1. : -1.;
                    for (int qf = 0; qf < nqf; ++qf)
                      {
                        const int    fq  = f * nqf + qf;
                        const double w   = w_f[fq];
                        const double x   = xi[qf * nf + m];
                        const double pj  = phi_f[fq * nb + aj];
                        const double E0n = W0n[fq];
                        const bool   cs_ = (flux == 0) || (flux == 2 && E0n > 0.);
                        double       v   = 0.;
                        if (b == 0)
                          v = (sj < DIM) ? eps * sg * pj : taus[f * 3] * pj;
                        else
                          {
                            const double mu  = (b == 1) ? mun : mup;
                            const double sgn = (b == 1) ? 1. : -1.;
                            if (bj == 0) // E, normal component
                              v = sgn * mu * sg * pj * (cs_ ? c0f[b * Fq + fq] : tr0[b * Fq + fq]);
                            else if (sj == DIM)
                              v = (cs_ ? sgn * mu * E0n : 0.) * pj - taus[f * 3 + b] * pj;
                            else
                              v = -U_T * mu * sg * pj;
                          }
                        s -= v * x * w;
                      }
                  }
                TC[idx] = s;
              }
            for (int idx = tid; idx < Nt * Nt; idx += T)
              {
                const int i = idx / Nt, j = idx % Nt;
                const int f = i / (ncomp * nf), ci = (i / nf) % ncomp, mi = i % nf;
                const int fj = j / (ncomp * nf), cj = (j / nf) % ncomp, mj = j % nf;
                const int b  = P.comps[ci];
                double    s  = 0.;
                if (f == fj && ci == cj && bcs[f * 3 + b] != 1.)
                  {
                    const double sign = (b == 0) ? -1. : 1.;
                    for (int qf = 0; qf < nqf; ++qf)
                      {
                        const int    fq  = f * nqf + qf;
                        const double E0n = W0n[fq];
                        const bool   upw = (flux == 1) || (flux == 2 && E0n <= 0.);
                        double       v   = sign * taus[f * 3 + b];
                        if (b != 0 && upw)
                          v += ((b == 1) ? mun : -mup) * E0n;
                        s += v * xi[qf * nf + mj] * xi[qf * nf + mi] * w_f[fq];
                      }
                  }
                TT[idx] = s;
              }
            // ------------- tt_rhs (T:1311-1447, T:1551-1588, Neumann T:1695-1734)
            for (int i = tid; i < Nt; i += T)
              {
                const int f = i / (ncomp * nf), ci = (i / nf) % ncomp, m = i % nf;
                const int b = P.comps[ci];
                double    s = 0.;
                const int bc = (int)bcs[f * 3 + b];
                if (bc != 1)
                  {
                    const int64_t Fi   = face_index(P, cell, f, DIM);
                    const double  sign = (b == 0) ? -1. : 1.;
                    const double  tau  = taus[f * 3 + b];
                    for (int qf = 0; qf < nqf; ++qf)
                      {
                        const int    fq  = f * nqf + qf;
                        const double E0n = W0n[fq];
                        const bool   cs_ = (flux == 0) || (flux == 2 && E0n > 0.);
                        double       term;
                        if (b == 0)
                          term = -eps * E0n - tau * c0f[fq];
                        else
                          {
                            const double mu  = (b == 1) ? mun : mup;
                            const double cst = cs_ ? c0f[b * Fq + fq] : tr0[b * Fq + fq];
                            term = ((b == 1) ? -1. : 1.) * cst * mu * E0n + U_T * mu * W0n[b * Fq + fq] +
                                   tau * c0f[b * Fq + fq];
                          }
                        term -= sign * tau * tr0[b * Fq + fq];
                        if (bc == 2 && !thermo)
                          term += P.face_bc_val[(Fi * 3 + b) * nqf + qf];
                        s += term * xi[qf * nf + m] * w_f[fq];
                      }
                  }
                TR[i] = s;
              }
          }
        __syncthreads();

        if (!recon)
          {
            // ------------- LocalCondenser::condense_ct_matrix (src/local_condenser.cpp:142-160)
            for (int i = tid; i < Nc; i += T)
              {
                double *row = A + i * ldA;
                double  r   = row[Nc];
                for (int j = 0; j < Nt; ++j)
                  if (dfl[j] != 0.)
                    {
                      r -= row[Nc + 1 + j] * dvl[j];
                      row[Nc + 1 + j] = 0.;
                    }
                row[Nc] = r;
              }
            __syncthreads();
          }

        if (mode == PlainProbe)
          {
            // get_local_cell_system (src/np_solver.cpp:2337-2445): the local
            // system before the Schur complement
            for (int idx = tid; idx < Nc * Nc; idx += T)
              if (A_.cc)
                A_.cc[wi * Nc * Nc + idx] = A[(idx / Nc) * ldA + idx % Nc];
            for (int idx = tid; idx < Nc * Nt; idx += T)
              if (A_.ct)
                A_.ct[wi * Nc * Nt + idx] = A[(idx / Nt) * ldA + Nc + 1 + idx % Nt];
            for (int idx = tid; idx < Nt * Nc; idx += T)
              if (A_.tc)
                A_.tc[wi * Nt * Nc + idx] = TC[idx];
            for (int idx = tid; idx < Nt * Nt; idx += T)
              if (A_.tt)
                A_.tt[wi * Nt * Nt + idx] = TT[idx];
            for (int i = tid; i < Nc; i += T)
              if (A_.c)
                A_.c[wi * Nc + i] = A[i * ldA + Nc];
            for (int i = tid; i < Nt; i += T)
              if (A_.t)
                A_.t[wi * Nt + i] = TR[i];
            __syncthreads();
            continue;
          }

        // ---------------- row equilibration and LU with partial pivoting of
        // cc applied to [cc_rhs | ct] (the Schur block, T:2651-2668)
        const int ncols = Nc + NR;
        for (int i = tid; i < Nc; i += T)
          {
            double mx = 0.;
            for (int j = 0; j < Nc; ++j)
              mx = fmax(mx, fabs(A[i * ldA + j]));
            rs[i] = mx > 0. ? 1. / mx : 1.;
          }
        __syncthreads();
        for (int idx = tid; idx < Nc * ncols; idx += T)
          {
            const int i = idx / ncols, j = idx % ncols;
            A[i * ldA + j] *= rs[i];
          }
        __syncthreads();
        bool singular = false;
        for (int k = 0; k < Nc; ++k)
          {
            if (tid < 32)
              {
                double best = -1.;
                int    bi   = k;
                for (int i = k + tid; i < Nc; i += 32)
                  {
                    const double v = fabs(A[i * ldA + k]);
                    if (v > best || (v != v))
                      {
                        best = (v != v) ? INFINITY : v;
                        bi   = i;
                      }
                  }
                for (int o = 16; o > 0; o >>= 1)
                  {
                    const double ob = __shfl_xor_sync(0xffffffffu, best, o);
                    const int    oi = __shfl_xor_sync(0xffffffffu, bi, o);
                    if (ob > best || (ob == best && oi < bi))
                      {
                        best = ob;
                        bi   = oi;
                      }
                  }
                if (tid == 0)
                  {
                    sh_piv  = bi;
                    sh_pmax = best;
                  }
              }
            __syncthreads();
            const int p = sh_piv;
            if (!(sh_pmax > 0.) || isinf(sh_pmax))
              {
                singular = true;
                break;
              }
            // a thread per column: row swap and rank-1 update of its own
            // columns (the columns left of k are eliminated and not needed)
            if (p != k)
              for (int jj = k + tid; jj < ncols; jj += T)
                {
                  const double t  = A[k * ldA + jj];
                  A[k * ldA + jj] = A[p * ldA + jj];
                  A[p * ldA + jj] = t;
                }
            __syncthreads();
            // rank-1 update: lanes over columns, warps over rows
            const double inv = 1. / A[k * ldA + k];
            for (int jj = k + 1 + (tid & 31); jj < ncols; jj += 32)
              {
                const double u = A[k * ldA + jj] * inv;
                if (u != 0.)
                  for (int ii = k + 1 + (tid >> 5); ii < Nc; ii += T / 32)
                    A[ii * ldA + jj] -= A[ii * ldA + k] * u;
              }
            __syncthreads();
          }
        if (singular)
          {
            if (tid == 0)
              atomicExch(P.status, 3);
            __syncthreads();
            continue;
          }
        // back substitution U X = Y: a warp per right-hand-side column,
        // lanes over the rows (no barrier between the steps)
        for (int jj = Nc + (tid >> 5); jj < ncols; jj += T / 32)
          for (int kk = Nc - 1; kk >= 0; --kk)
            {
              const double x = A[kk * ldA + jj] / A[kk * ldA + kk];
              __syncwarp();
              if ((tid & 31) == 0)
                A[kk * ldA + jj] = x;
              if (x != 0.)
                for (int ii = tid & 31; ii < kk; ii += 32)
                  A[ii * ldA + jj] -= A[ii * ldA + kk] * x;
              __syncwarp();
            }
        __syncthreads();

        if (recon)
          {
            // the cell update of the enabled components (T:2688-2697)
            double *out = A_.update_cell + cell * NCA;
            for (int i = tid; i < NCA; i += T)
              {
                const int ce = ce_of[i / ((DIM + 1) * nb)];
                out[i]       = ce >= 0 ? A[(ce * (DIM + 1) * nb + i % ((DIM + 1) * nb)) * ldA + Nc] : 0.;
              }
            __syncthreads();
            continue;
          }

        // ---------------- Schur complement: tt += tc X_t, tt_rhs += tc X_0
        for (int idx = tid; idx < Nt * NR; idx += T)
          {
            const int i = idx / NR, j = idx % NR;
            double    s = 0.;
            for (int l = 0; l < Nc; ++l)
              s += TC[i * Nc + l] * A[l * ldA + Nc + j];
            if (j == 0)
              P.rhs[cell * Nt + i] = TR[i] + s;
            else
              P.tt[(cell * Nt + i) * Nt + (j - 1)] = TT[i * Nt + (j - 1)] + s;
          }
        for (int i = tid; i < Nt; i += T)
          {
            P.dflag[cell * Nt + i] = dfl[i] != 0. ? 1 : 0;
            P.dval[cell * Nt + i]  = dvl[i];
          }
        __syncthreads();
      }
  }
} // namespace ddhdg
