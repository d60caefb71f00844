// Device kernels of the HDG hot path (sm_100a, FP64).
//
// One warp condenses one cell; a CTA holds several warps that share the
// constant basis / elimination tables staged in shared memory, and the grid is
// persistent (a multiple of the SM count) with a stride loop over cells.
//
// Per cell the kernel restates the reference's local system
// (include/assembling_methods.template.h:269-2160) in block form: the flux
// unknowns (E, Wn, Wp) are eliminated through the constant mass matrix
// (tables P, Q), which leaves the scalar system S y = R of size
// ncomp*(k+1)^d with right-hand sides [residual | one column per trace dof].
// S is row-equilibrated and LU-factorised with partial pivoting; the
// condensed trace system tt + tc cc^-1 [ct | rhs]
// (include/assembling_methods.template.h:2651-2686) is evaluated as face
// integrals of the solved columns.  The solved columns are kept for the
// reconstruction (include/assembling_methods.template.h:2688-2697), which then
// needs no second assembly or factorisation.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace ddhdg
{
  constexpr double KB_ = 1.380649E-23;
  constexpr double Q_  = 1.602176634E-19;
  constexpr double EV_ = 1.602176565E-19;

  // offsets (in doubles) of the tables inside the staged table block
  struct TabOff
  {
    int phi_c, grad_c, w_c, phi_f, w_f, xi, fminvw, PW_c, PW_f, QW_c, QW_f, P,
      Q, minv, total;
  };

  struct KParams
  {
    // mesh
    int     n[3];
    int64_t ncells;
    int64_t face_off[3];
    int     face_ext[3][3];
    // tables (device, global) and their layout
    const double *tables;
    TabOff        to;
    // physics (rescaled)
    double eps, mun, mup, U_T, T, V_rescale, n_rescale, rec_rescale;
    double nc, nv, ec, ev; // ec, ev in joule
    int    rec_type;
    double srh_ni, srh_tau_n, srh_tau_p;
    const double *rec_a, *rec_b, *rec_c, *doping, *tau_table;
    double        tau[3];
    const int32_t *face_bc;
    const double  *face_bc_val;
    // mode
    int comps[3], ncomp, flux, phi_linearize, thermo, jfix;
    int ncol;  // columns of the scalar system: 1 + Nt (+ Nt)
    int ycols; // columns kept for the reconstruction: 1 + Nt
    int wpb;   // warps per block
    int chunk; // columns per chunk in the condensation stage
    int stage; // 1: copy the tables to shared memory, 0: read them from L1/L2
    // state
    const double *cell_state, *trace_state;
    // outputs
    double  *tt, *rhs, *dval, *ycache;
    int32_t *dflag;
    int     *status;
  };

  template <int DIM, int K>
  struct Dims
  {
    static constexpr int ipow(int b, int e) { return e == 0 ? 1 : b * ipow(b, e - 1); }
    static constexpr int nb     = ipow(K + 1, DIM);
    static constexpr int nf     = ipow(K + 1, DIM - 1);
    static constexpr int nqc    = nb;
    static constexpr int nqf    = nf;
    static constexpr int F      = 2 * DIM;
    static constexpr int Nc_all = 3 * (DIM + 1) * nb;
  };

  // Per-warp workspace layout (doubles), shared by host and device.
  struct WsOff
  {
    int coef, lam, c0, W0, qc, c0f, W0n, tr0, Wrc, Wrf, tau, S, R, g, rhsA,
      colf, total;
  };

  __host__ __device__ inline WsOff
  ws_layout(int dim, int nb, int nf, int ncomp, int ncol, int chunk)
  {
    const int F = 2 * dim, nqc = nb, nqf = nf;
    const int Ns = ncomp * nb, Nt = F * ncomp * nf;
    WsOff     o;
    int       p = 0;
    o.coef      = p;
    p += 3 * (dim + 1) * nb;
    o.lam = p;
    p += F * 3 * nf;
    o.c0 = p;
    p += 3 * nqc;
    o.W0 = p;
    p += 3 * dim * nqc;
    o.qc = p;
    p += 6 * nqc;
    o.c0f = p;
    p += 3 * F * nqf;
    o.W0n = p;
    p += 3 * F * nqf;
    o.tr0 = p;
    p += 3 * F * nqf;
    o.Wrc = p;
    p += 3 * dim * nqc;
    o.Wrf = p;
    p += 3 * F * nqf;
    o.tau = p;
    p += F * 3 + F * 3; // tau values, then bc types (stored as doubles)
    o.S = p;
    p += Ns * (Ns + 1);
    o.R = p;
    p += Ns * ncol;
    o.g = p;
    p += Nt;
    o.rhsA = p;
    p += 2 * Nt;
    o.colf = p;
    p += chunk * ncomp * F * nqf * 2;
    p       = (p + 1) & ~1; // 16-byte multiple
    o.total = p;
    return o;
  }

  __device__ inline int64_t
  face_index(const KParams &P, int64_t cell, int f, int dim)
  {
    int ci[3];
    ci[0]       = (int)(cell % P.n[0]);
    ci[1]       = (int)((cell / P.n[0]) % P.n[1]);
    ci[2]       = (int)(cell / ((int64_t)P.n[0] * P.n[1]));
    const int a = f / 2;
    ci[a] += f % 2;
    int64_t idx = 0, stride = 1;
    for (int b = 0; b < dim; ++b)
      {
        idx += ci[b] * stride;
        stride *= P.face_ext[a][b];
      }
    return P.face_off[a] + idx;
  }

  // ------------------------------------------------------------ condense
  template <int DIM, int K>
  __global__ void __launch_bounds__(256)
  condense_kernel(const KParams P)
  {
    using Dm           = Dims<DIM, K>;
    constexpr int nb   = Dm::nb;
    constexpr int nf   = Dm::nf;
    constexpr int nqc  = Dm::nqc;
    constexpr int nqf  = Dm::nqf;
    constexpr int F    = Dm::F;
    constexpr int NCA  = Dm::Nc_all;
    extern __shared__ double smem[];

    const int lane  = threadIdx.x & 31;
    const int warp  = threadIdx.x >> 5;
    const int ncomp = P.ncomp;
    const int Ns    = ncomp * nb;
    const int Nt    = F * ncomp * nf;
    const int ncol  = P.ncol;
    const int ldS   = Ns + 1;
    const int CH    = P.chunk;

    // ---- stage the tables (shared by every warp of the CTA)
    const double *tb = P.tables;
    if (P.stage)
      {
        for (int i = threadIdx.x; i < P.to.total; i += blockDim.x)
          smem[i] = P.tables[i];
        __syncthreads();
        tb = smem;
      }
    const double *phi_c  = tb + P.to.phi_c;
    const double *grad_c = tb + P.to.grad_c;
    const double *w_c    = tb + P.to.w_c;
    const double *phi_f  = tb + P.to.phi_f;
    const double *w_f    = tb + P.to.w_f;
    const double *xi     = tb + P.to.xi;
    const double *fminvw = tb + P.to.fminvw;
    const double *PW_c   = tb + P.to.PW_c;
    const double *PW_f   = tb + P.to.PW_f;
    const double *QW_c   = tb + P.to.QW_c;
    const double *QW_f   = tb + P.to.QW_f;

    const WsOff wo = ws_layout(DIM, nb, nf, ncomp, ncol, CH);
    double     *ws = smem + (P.stage ? ((P.to.total + 1) & ~1) : 0) + warp * wo.total;
    double *coef = ws + wo.coef, *lam = ws + wo.lam, *c0 = ws + wo.c0,
           *W0 = ws + wo.W0, *qc = ws + wo.qc, *c0f = ws + wo.c0f,
           *W0n = ws + wo.W0n, *tr0 = ws + wo.tr0, *Wrc = ws + wo.Wrc,
           *Wrf = ws + wo.Wrf, *taus = ws + wo.tau, *bcs = ws + wo.tau + F * 3,
           *S = ws + wo.S, *R = ws + wo.R, *gv = ws + wo.g,
           *rhsA = ws + wo.rhsA, *colf = ws + wo.colf;

    const double eps = P.eps, mun = P.mun, mup = P.mup, U_T = P.U_T;
    const bool   thermo   = P.thermo != 0;
    const bool   phi_mode = thermo || P.phi_linearize;
    const double ds       = (P.jfix & 1) ? -1. : 1.;
    const int    flux     = P.flux;

    for (int64_t cell = (int64_t)blockIdx.x * P.wpb + warp; cell < P.ncells;
         cell += (int64_t)gridDim.x * P.wpb)
      {
        // ---------------------------------------------- load the state
        const double *cs = P.cell_state + cell * NCA;
        for (int i = lane; i < NCA; i += 32)
          coef[i] = cs[i];
        for (int i = lane; i < F * 3 * nf; i += 32)
          {
            const int     f  = i / (3 * nf);
            const int64_t Fi = face_index(P, cell, f, DIM);
            lam[i]           = P.trace_state[Fi * 3 * nf + (i % (3 * nf))];
          }
        for (int i = lane; i < F * 3; i += 32)
          {
            const int     f  = i / 3;
            const int     b  = i % 3;
            const int64_t Fi = face_index(P, cell, f, DIM);
            taus[i] = P.tau_table ? P.tau_table[(cell * F + f) * 3 + b] : P.tau[b];
            bcs[i]  = (double)P.face_bc[Fi * 3 + b];
          }
        __syncwarp();

        // ------------------------------- previous fields at quadrature pts
        for (int i = lane; i < 3 * (DIM + 1) * nqc; i += 32)
          {
            const int b = i / ((DIM + 1) * nqc);
            const int s = (i / nqc) % (DIM + 1);
            const int q = i % nqc;
            double    v = 0.;
            const double *cf = coef + (b * (DIM + 1) + s) * nb;
#pragma unroll
            for (int a = 0; a < nb; ++a)
              v += phi_c[q * nb + a] * cf[a];
            if (s < DIM)
              W0[(b * DIM + s) * nqc + q] = v;
            else
              c0[b * nqc + q] = v;
          }
        for (int i = lane; i < 3 * F * nqf; i += 32)
          {
            const int     b  = i / (F * nqf);
            const int     f  = (i / nqf) % F;
            const int     qf = i % nqf;
            const int     ax = f / 2;
            const double  sg = (f & 1) ? 1. : -1.;
            const double *ph = phi_f + (f * nqf + qf) * nb;
            const double *cS = coef + (b * (DIM + 1) + DIM) * nb;
            const double *cW = coef + (b * (DIM + 1) + ax) * nb;
            double        u = 0., wn = 0.;
#pragma unroll
            for (int a = 0; a < nb; ++a)
              {
                u += ph[a] * cS[a];
                wn += ph[a] * cW[a];
              }
            double t = 0.;
#pragma unroll
            for (int m = 0; m < nf; ++m)
              t += xi[qf * nf + m] * lam[(f * 3 + b) * nf + m];
            c0f[i] = u;
            W0n[i] = sg * wn;
            tr0[i] = t;
          }
        __syncwarp();

        // ----------------------------- coefficients at cell quadrature pts
        bool nen = false, pen = false;
        for (int c = 0; c < ncomp; ++c)
          {
            nen |= P.comps[c] == 1;
            pen |= P.comps[c] == 2;
          }
        for (int q = lane; q < nqc; q += 32)
          {
            const double n0 = c0[nqc + q], p0 = c0[2 * nqc + q],
                         V0 = c0[q];
            double r = 0., drn = 0., drp = 0.;
            if (nen || pen)
              {
                const double rf = P.n_rescale;
                if (P.rec_type == 1)
                  {
                    const double ni  = P.srh_ni / rf;
                    const double num = n0 * p0 - ni * ni;
                    const double den =
                      P.srh_tau_p * (n0 + ni) + P.srh_tau_n * (p0 + ni);
                    r   = num * rf / den;
                    drn = p0 / den - num * P.srh_tau_p / (den * den);
                    drp = n0 / den - num * P.srh_tau_n / (den * den);
                  }
                else
                  {
                    const int64_t idx = cell * nqc + q;
                    const double  a_  = P.rec_a ? P.rec_a[idx] : 0.;
                    const double  b_  = P.rec_b ? P.rec_b[idx] : 0.;
                    const double  c_  = P.rec_c ? P.rec_c[idx] : 0.;
                    r                 = a_ + (b_ * n0 + c_ * p0) * rf;
                    drn               = b_;
                    drp               = c_;
                  }
                r /= P.rec_rescale;
                drn /= P.rec_rescale;
                drp /= P.rec_rescale;
                if (P.jfix & 2)
                  {
                    drn *= rf;
                    drp *= rf;
                  }
              }
            double phider = 0., phirhs = 0.;
            if (phi_mode)
              {
                const double KbT = KB_ * P.T / (Q_ * P.V_rescale);
                const double evr = P.ev / (Q_ * P.V_rescale);
                const double ecr = P.ec / (Q_ * P.V_rescale);
                double       phn = 0., php = 0.;
                if (!thermo)
                  {
                    // quasi Fermi potentials (include/solver.h:343-376)
                    const double U = P.T * (KB_ / Q_);
                    const double Vp = V0 * P.V_rescale;
                    phn = (Vp - P.ec / Q_ - U * log(n0 * P.n_rescale / P.nc)) /
                          P.V_rescale;
                    php = (Vp - P.ev / Q_ + U * log(p0 * P.n_rescale / P.nv)) /
                          P.V_rescale;
                    // only the enabled carriers are linearised
                    if (!nen)
                      phn = 0.;
                    if (!pen)
                      php = 0.;
                  }
                const double e1 = exp((evr - V0 + php) / KbT);
                const double e2 = exp((V0 - phn - ecr) / KbT);
                phider = -1. / P.n_rescale * (P.nv / KbT * e1 + P.nc / KbT * e2);
                phirhs = 1. / P.n_rescale * (P.nv * e1 - P.nc * e2);
              }
            qc[0 * nqc + q] = r;
            qc[1 * nqc + q] = drn;
            qc[2 * nqc + q] = drp;
            qc[3 * nqc + q] = phider;
            qc[4 * nqc + q] = phirhs;
            qc[5 * nqc + q] = P.doping[cell * nqc + q];
          }

        // ---------------- flux residual field W = P u0 - W0 - Q lam0 (per comp)
        for (int i = lane; i < ncomp * DIM * nqc; i += 32)
          {
            const int ce = i / (DIM * nqc);
            const int b  = P.comps[ce];
            const int s  = (i / nqc) % DIM;
            const int q  = i % nqc;
            const double *cS = coef + (b * (DIM + 1) + DIM) * nb;
            double        v  = -W0[(b * DIM + s) * nqc + q];
#pragma unroll
            for (int e = 0; e < nb; ++e)
              v += PW_c[(e * nqc + q) * DIM + s] * cS[e];
            for (int t = 0; t < F * nf; ++t)
              v -= QW_c[(t * nqc + q) * DIM + s] *
                   lam[((t / nf) * 3 + b) * nf + (t % nf)];
            Wrc[(ce * DIM + s) * nqc + q] = v;
          }
        for (int i = lane; i < ncomp * F * nqf; i += 32)
          {
            const int ce = i / (F * nqf);
            const int b  = P.comps[ce];
            const int f  = (i / nqf) % F;
            const int qf = i % nqf;
            const double *cS = coef + (b * (DIM + 1) + DIM) * nb;
            double        v  = -W0n[(b * F + f) * nqf + qf];
#pragma unroll
            for (int e = 0; e < nb; ++e)
              v += PW_f[(e * F + f) * nqf + qf] * cS[e];
            for (int t = 0; t < F * nf; ++t)
              v -= QW_f[(t * F + f) * nqf + qf] *
                   lam[((t / nf) * 3 + b) * nf + (t % nf)];
            Wrf[(ce * F + f) * nqf + qf] = v;
          }
        __syncwarp();

        // --------------------------------------------- Dirichlet increments
        for (int t = lane; t < Nt; t += 32)
          {
            const int f  = t / (ncomp * nf);
            const int ce = (t / nf) % ncomp;
            const int m  = t % nf;
            const int b  = P.comps[ce];
            double    g  = 0.;
            if (bcs[f * 3 + b] == 1.)
              {
                if (!thermo)
                  {
                    const int64_t Fi = face_index(P, cell, f, DIM);
                    for (int qf = 0; qf < nqf; ++qf)
                      g += fminvw[m * nqf + qf] *
                           (P.face_bc_val[(Fi * 3 + b) * nqf + qf] -
                            tr0[(b * F + f) * nqf + qf]);
                  }
                rhsA[Nt + t] = 1.; // flag
              }
            else
              rhsA[Nt + t] = 0.;
            gv[t] = g;
          }

        // ------------------------------------------------- scalar system S
        for (int idx = lane; idx < Ns * Ns; idx += 32)
          {
            const int i  = idx / Ns;
            const int j  = idx % Ns;
            const int b  = P.comps[i / nb];
            const int bp = P.comps[j / nb];
            const int a  = i % nb;
            const int e  = j % nb;
            double    v  = 0.;
            for (int q = 0; q < nqc; ++q)
              {
                const double pa = phi_c[q * nb + a];
                const double pe = phi_c[q * nb + e];
                const double *ga = grad_c + (q * nb + a) * DIM;
                const double *pw = PW_c + (e * nqc + q) * DIM;
                double        alpha = 0., kappa = 0., gdotpw = 0., bterm = 0.;
#pragma unroll
                for (int s = 0; s < DIM; ++s)
                  gdotpw += ga[s] * pw[s];
                if (b == 0)
                  {
                    if (bp == 0)
                      {
                        alpha = phi_mode ? -qc[3 * nqc + q] : 0.;
                        kappa = -eps;
                      }
                    else if (!phi_mode)
                      alpha = (bp == 1) ? 1. : -1.;
                  }
                else
                  {
                    const double *E0 = W0; // E0[s*nqc + q]
                    if (bp == 0)
                      kappa = (b == 1) ? ds * c0[nqc + q] * mun :
                                         -ds * c0[2 * nqc + q] * mup;
                    else
                      {
                        alpha = (bp == 1) ? -qc[nqc + q] : -qc[2 * nqc + q];
                        if (bp == b)
                          {
                            kappa     = U_T * ((b == 1) ? mun : mup);
                            const double sg = (b == 1) ? -mun : mup;
                            double       eg = 0.;
#pragma unroll
                            for (int s = 0; s < DIM; ++s)
                              eg += E0[s * nqc + q] * ga[s];
                            bterm = sg * eg;
                          }
                      }
                  }
                v += w_c[q] * (alpha * pa * pe + bterm * pe + kappa * gdotpw);
              }
            for (int f = 0; f < F; ++f)
              for (int qf = 0; qf < nqf; ++qf)
                {
                  const double pa = phi_f[(f * nqf + qf) * nb + a];
                  if (pa == 0.)
                    continue;
                  const double pe  = phi_f[(f * nqf + qf) * nb + e];
                  const double pwf = PW_f[(e * F + f) * nqf + qf];
                  const int    fq  = f * nqf + qf;
                  const double E0n = W0n[fq];
                  const bool   cellside =
                    (flux == 0) || (flux == 2 && E0n > 0.);
                  const double tb_ = taus[f * 3 + b];
                  double       gamma = 0., rho = 0.;
                  if (b == 0)
                    {
                      if (bp == 0)
                        {
                          gamma = tb_;
                          rho   = eps;
                        }
                    }
                  else if (b == 1)
                    {
                      if (bp == 0)
                        rho = mun * (cellside ? c0f[F * nqf + fq] : tr0[F * nqf + fq]);
                      else if (bp == 1)
                        {
                          gamma = (cellside ? mun * E0n : 0.) - tb_;
                          rho   = -U_T * mun;
                        }
                    }
                  else
                    {
                      if (bp == 0)
                        rho = -mup * (cellside ? c0f[2 * F * nqf + fq] :
                                                 tr0[2 * F * nqf + fq]);
                      else if (bp == 2)
                        {
                          gamma = (cellside ? -mup * E0n : 0.) - tb_;
                          rho   = -U_T * mup;
                        }
                    }
                  v += w_f[fq] * pa * (gamma * pe + rho * pwf);
                }
            S[i * ldS + j] = v;
          }

        // ----------------------------------------- right-hand sides R
        for (int idx = lane; idx < Ns * ncol; idx += 32)
          {
            const int i   = idx / ncol;
            const int col = idx % ncol;
            const int b   = P.comps[i / nb];
            const int a   = i % nb;
            double    v   = 0.;
            if (col == 0)
              {
                // residual rows minus the flux-elimination term A_zW Wres
                for (int q = 0; q < nqc; ++q)
                  {
                    const double  pa = phi_c[q * nb + a];
                    const double *ga = grad_c + (q * nb + a) * DIM;
                    const double  V0 = c0[q], n0 = c0[nqc + q], p0 = c0[2 * nqc + q];
                    double        r  = 0.;
                    if (b == 0)
                      {
                        double eg = 0.;
#pragma unroll
                        for (int s = 0; s < DIM; ++s)
                          eg += W0[s * nqc + q] * ga[s];
                        r = eps * eg + qc[5 * nqc + q] * pa +
                            (phi_mode ? qc[4 * nqc + q] : (p0 - n0)) * pa;
                      }
                    else
                      {
                        const double mu = (b == 1) ? mun : mup;
                        const double cb = (b == 1) ? n0 : -p0;
                        double       jg = 0.;
#pragma unroll
                        for (int s = 0; s < DIM; ++s)
                          jg += (cb * mu * W0[s * nqc + q] -
                                 U_T * mu * W0[(b * DIM + s) * nqc + q]) *
                                ga[s];
                        r = qc[q] * pa + jg;
                      }
                    // - sum_b' kappa_{b b'} grad(pa) . Wres_b'
                    for (int ce = 0; ce < ncomp; ++ce)
                      {
                        const int bp    = P.comps[ce];
                        double    kappa = 0.;
                        if (b == 0 && bp == 0)
                          kappa = -eps;
                        else if (b != 0 && bp == 0)
                          kappa = (b == 1) ? ds * n0 * mun : -ds * p0 * mup;
                        else if (b != 0 && bp == b)
                          kappa = U_T * ((b == 1) ? mun : mup);
                        if (kappa != 0.)
                          {
                            double gw = 0.;
#pragma unroll
                            for (int s = 0; s < DIM; ++s)
                              gw += ga[s] * Wrc[(ce * DIM + s) * nqc + q];
                            r -= kappa * gw;
                          }
                      }
                    v += w_c[q] * r;
                  }
                for (int f = 0; f < F; ++f)
                  for (int qf = 0; qf < nqf; ++qf)
                    {
                      const double pa = phi_f[(f * nqf + qf) * nb + a];
                      if (pa == 0.)
                        continue;
                      const int    fq  = f * nqf + qf;
                      const double E0n = W0n[fq];
                      const bool   cellside =
                        (flux == 0) || (flux == 2 && E0n > 0.);
                      const double tb_ = taus[f * 3 + b];
                      double       r   = 0.;
                      const double cb0 = c0f[b * F * nqf + fq];
                      const double tb0 = tr0[b * F * nqf + fq];
                      if (b == 0)
                        r = tb_ * tb0 - eps * E0n - tb_ * cb0;
                      else
                        {
                          const double mu   = (b == 1) ? mun : mup;
                          const double sg   = (b == 1) ? 1. : -1.;
                          const double cstr = cellside ? cb0 : tb0;
                          const double Jf =
                            sg * cstr * mu * E0n - U_T * mu * W0n[b * F * nqf + fq];
                          r = -tb_ * tb0 - Jf + tb_ * cb0;
                        }
                      for (int ce = 0; ce < ncomp; ++ce)
                        {
                          const int bp  = P.comps[ce];
                          double    rho = 0.;
                          if (b == 0 && bp == 0)
                            rho = eps;
                          else if (b != 0 && bp == 0)
                            rho = (b == 1) ? mun * (cellside ? cb0 : tb0) :
                                             -mup * (cellside ? cb0 : tb0);
                          else if (b != 0 && bp == b)
                            rho = -U_T * ((b == 1) ? mun : mup);
                          r -= rho * Wrf[(ce * F + f) * nqf + qf];
                        }
                      v += w_f[fq] * pa * r;
                    }
              }
            else
              {
                const bool drift_col = col > Nt;
                const int  t         = drift_col ? col - 1 - Nt : col - 1;
                const int  ft        = t / (ncomp * nf);
                const int  cet       = (t / nf) % ncomp;
                const int  mt        = t % nf;
                const int  bp        = P.comps[cet];
                if (!drift_col)
                  {
                    // ct_z (no drift) - A_zW Q_t
                    if (bp == b)
                      {
                        const double tb_ = taus[ft * 3 + b];
                        const double cc_ = (b == 0) ? -tb_ : tb_;
                        for (int qf = 0; qf < nqf; ++qf)
                          v += w_f[ft * nqf + qf] * cc_ * xi[qf * nf + mt] *
                               phi_f[(ft * nqf + qf) * nb + a];
                      }
                    for (int q = 0; q < nqc; ++q)
                      {
                        double kappa = 0.;
                        if (b == 0 && bp == 0)
                          kappa = -eps;
                        else if (b != 0 && bp == 0)
                          kappa = (b == 1) ? ds * c0[nqc + q] * mun :
                                             -ds * c0[2 * nqc + q] * mup;
                        else if (b != 0 && bp == b)
                          kappa = U_T * ((b == 1) ? mun : mup);
                        if (kappa == 0.)
                          continue;
                        const double *ga = grad_c + (q * nb + a) * DIM;
                        const double *qw = QW_c + ((ft * nf + mt) * nqc + q) * DIM;
                        double        gw = 0.;
#pragma unroll
                        for (int s = 0; s < DIM; ++s)
                          gw += ga[s] * qw[s];
                        v -= w_c[q] * kappa * gw;
                      }
                    for (int f = 0; f < F; ++f)
                      for (int qf = 0; qf < nqf; ++qf)
                        {
                          const double pa = phi_f[(f * nqf + qf) * nb + a];
                          if (pa == 0.)
                            continue;
                          const int    fq  = f * nqf + qf;
                          const double E0n = W0n[fq];
                          const bool   cellside =
                            (flux == 0) || (flux == 2 && E0n > 0.);
                          double rho = 0.;
                          if (b == 0 && bp == 0)
                            rho = eps;
                          else if (b != 0 && bp == 0)
                            {
                              const double cstr = cellside ? c0f[b * F * nqf + fq] :
                                                             tr0[b * F * nqf + fq];
                              rho = (b == 1) ? mun * cstr : -mup * cstr;
                            }
                          else if (b != 0 && bp == b)
                            rho = -U_T * ((b == 1) ? mun : mup);
                          if (rho != 0.)
                            v -= w_f[fq] * rho * pa *
                                 QW_f[((ft * nf + mt) * F + f) * nqf + qf];
                        }
                  }
                else if (bp == b && b != 0)
                  {
                    // drift part of ct (use_trace / Qiu-Shi upwind faces)
                    for (int qf = 0; qf < nqf; ++qf)
                      {
                        const int    fq  = ft * nqf + qf;
                        const double E0n = W0n[fq];
                        const bool   drift =
                          (flux == 1) || (flux == 2 && E0n <= 0.);
                        if (!drift)
                          continue;
                        const double cc_ = (b == 1) ? mun * E0n : -mup * E0n;
                        v += w_f[fq] * cc_ * xi[qf * nf + mt] *
                             phi_f[(ft * nqf + qf) * nb + a];
                      }
                  }
              }
            R[i * ncol + col] = v;
          }
        __syncwarp();

        // ------------------------------ equilibrate rows, LU with pivoting
        for (int i = lane; i < Ns; i += 32)
          {
            double mx = 0.;
            for (int j = 0; j < Ns; ++j)
              mx = fmax(mx, fabs(S[i * ldS + j]));
            const double sc = (mx > 0.) ? 1. / mx : 1.;
            for (int j = 0; j < Ns; ++j)
              S[i * ldS + j] *= sc;
            for (int c = 0; c < ncol; ++c)
              R[i * ncol + c] *= sc;
          }
        __syncwarp();
        bool singular = false;
        for (int j = 0; j < Ns; ++j)
          {
            // pivot search over rows j..Ns-1
            double best = -1.;
            int    bi   = j;
            for (int i = j + lane; i < Ns; i += 32)
              {
                const double v = fabs(S[i * ldS + j]);
                if (v > best)
                  {
                    best = v;
                    bi   = i;
                  }
              }
#pragma unroll
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
            if (!(best > 0.) || !isfinite(best))
              singular = true;
            if (bi != j)
              {
                for (int c = lane; c < Ns; c += 32)
                  {
                    const double t0 = S[j * ldS + c];
                    S[j * ldS + c]  = S[bi * ldS + c];
                    S[bi * ldS + c] = t0;
                  }
                for (int c = lane; c < ncol; c += 32)
                  {
                    const double t0 = R[j * ncol + c];
                    R[j * ncol + c] = R[bi * ncol + c];
                    R[bi * ncol + c] = t0;
                  }
              }
            __syncwarp();
            const double piv = S[j * ldS + j];
            const double inv = (piv != 0.) ? 1. / piv : 0.;
            for (int i = j + 1 + lane; i < Ns; i += 32)
              S[i * ldS + j] *= inv;
            __syncwarp();
            const int nrow = Ns - j - 1;
            const int wS   = Ns - j - 1;
            const int wtot = wS + ncol;
            for (int idx = lane; idx < nrow * wtot; idx += 32)
              {
                const int    i = j + 1 + idx / wtot;
                const int    c = idx % wtot;
                const double l = S[i * ldS + j];
                if (c < wS)
                  S[i * ldS + j + 1 + c] -= l * S[j * ldS + j + 1 + c];
                else
                  R[i * ncol + (c - wS)] -= l * R[j * ncol + (c - wS)];
              }
            __syncwarp();
          }
        // back substitution (R becomes Y)
        for (int j = Ns - 1; j >= 0; --j)
          {
            const double piv = S[j * ldS + j];
            const double inv = (piv != 0.) ? 1. / piv : 0.;
            for (int c = lane; c < ncol; c += 32)
              R[j * ncol + c] *= inv;
            __syncwarp();
            for (int idx = lane; idx < j * ncol; idx += 32)
              {
                const int i = idx / ncol;
                const int c = idx % ncol;
                R[i * ncol + c] -= S[i * ldS + j] * R[j * ncol + c];
              }
            __syncwarp();
          }
        if (singular && lane == 0)
          atomicExch(P.status, 3);

        // ----------------------------- keep Y for the reconstruction
        {
          // column-major [col][row] so that both kernels stream it coalesced
          double *yc = P.ycache + cell * (int64_t)Ns * P.ycols;
          for (int idx = lane; idx < Ns * P.ycols; idx += 32)
            {
              const int i = idx % Ns;
              const int c = idx / Ns;
              yc[idx]     = R[i * ncol + c];
            }
        }

        // --------------------- condensation: tc * [Y0 | Y_t] on the faces
        for (int i = lane; i < Nt; i += 32)
          rhsA[i] = 0.;
        double *tt_out = P.tt + cell * (int64_t)Nt * Nt;
        const int ncolc = 1 + Nt; // output columns (drift folded in)
        for (int c0_ = 0; c0_ < ncolc; c0_ += CH)
          {
            const int nch = min(CH, ncolc - c0_);
            // column fields on the faces: scalar of comp ce and flux normal
            const int per = ncomp * F * nqf;
            for (int idx = lane; idx < nch * per; idx += 32)
              {
                const int cc  = idx / per;
                const int col = c0_ + cc;
                const int r   = idx % per;
                const int ce  = r / (F * nqf);
                const int f   = (r / nqf) % F;
                const int qf  = r % nqf;
                const int fq  = f * nqf + qf;
                double    u = 0., wn = 0.;
                // base part of the flux field
                if (col == 0)
                  wn = Wrf[(ce * F + f) * nqf + qf];
                else
                  {
                    const int t  = col - 1;
                    const int ft = t / (ncomp * nf);
                    const int ct = (t / nf) % ncomp;
                    const int mt = t % nf;
                    if (ct == ce)
                      wn = QW_f[((ft * nf + mt) * F + f) * nqf + qf];
                  }
                const bool   two = (col > 0) && (ncol > 1 + Nt);
#pragma unroll
                for (int e = 0; e < nb; ++e)
                  {
                    double y = R[(ce * nb + e) * ncol + col];
                    if (two)
                      y += R[(ce * nb + e) * ncol + col + Nt];
                    u += phi_f[fq * nb + e] * y;
                    wn += PW_f[(e * F + f) * nqf + qf] * y;
                  }
                colf[(cc * per + r) * 2 + 0] = u;
                colf[(cc * per + r) * 2 + 1] = wn;
              }
            __syncwarp();
            for (int i = lane; i < Nt; i += 32)
              {
                const int fi  = i / (ncomp * nf);
                const int cei = (i / nf) % ncomp;
                const int mi  = i % nf;
                const int b   = P.comps[cei];
                const bool rowD = rhsA[Nt + i] != 0.;
                for (int cc = 0; cc < nch; ++cc)
                  {
                    const int col = c0_ + cc;
                    double    x   = 0.;
                    if (!rowD)
                      for (int qf = 0; qf < nqf; ++qf)
                        {
                          const int    fq  = fi * nqf + qf;
                          const double E0n = W0n[fq];
                          const bool   cellside =
                            (flux == 0) || (flux == 2 && E0n > 0.);
                          const double tb_ = taus[fi * 3 + b];
                          const double *cf = colf + (cc * ncomp * F * nqf) * 2;
                          const double u   = cf[((cei * F + fi) * nqf + qf) * 2 + 0];
                          double       val;
                          if (b == 0)
                            val = -tb_ * u;
                          else if (b == 1)
                            val = (-(cellside ? mun * E0n : 0.) + tb_) * u;
                          else
                            val = ((cellside ? mup * E0n : 0.) + tb_) * u;
                          for (int ce = 0; ce < ncomp; ++ce)
                            {
                              const int bp = P.comps[ce];
                              double    cw = 0.;
                              if (b == 0 && bp == 0)
                                cw = -eps;
                              else if (b != 0 && bp == 0)
                                {
                                  const double cstr = cellside ?
                                                        c0f[b * F * nqf + fq] :
                                                        tr0[b * F * nqf + fq];
                                  cw = (b == 1) ? -cstr * mun : cstr * mup;
                                }
                              else if (b != 0 && bp == b)
                                cw = U_T * ((b == 1) ? mun : mup);
                              if (cw != 0.)
                                val += cw * cf[((ce * F + fi) * nqf + qf) * 2 + 1];
                            }
                          x += w_f[fq] * xi[qf * nf + mi] * val;
                        }
                    if (col == 0)
                      rhsA[i] += x;
                    else
                      {
                        const int t = col - 1;
                        if (rhsA[Nt + t] != 0.)
                          {
                            rhsA[i] -= x * gv[t];
                            tt_out[(int64_t)i * Nt + t] = 0.;
                          }
                        else
                          {
                            // face part of tt (same face and component)
                            double tf = 0.;
                            const int ft  = t / (ncomp * nf);
                            const int cet = (t / nf) % ncomp;
                            if (!rowD && ft == fi && cet == cei)
                              {
                                const int    mt  = t % nf;
                                const double sgn = (b == 0) ? -1. : 1.;
                                for (int qf = 0; qf < nqf; ++qf)
                                  {
                                    const int    fq  = fi * nqf + qf;
                                    const double E0n = W0n[fq];
                                    double       cf_ = sgn * taus[fi * 3 + b];
                                    if (b != 0 && ((flux == 1) || (flux == 2 && E0n <= 0.)))
                                      cf_ += (b == 1) ? mun * E0n : -mup * E0n;
                                    tf += w_f[fq] * cf_ * xi[qf * nf + mi] *
                                          xi[qf * nf + mt];
                                  }
                              }
                            tt_out[(int64_t)i * Nt + t] = rowD ? 0. : tf + x;
                          }
                      }
                  }
              }
            __syncwarp();
          }

        // ------------------------------------------ face part of the rhs
        for (int i = lane; i < Nt; i += 32)
          {
            const int  fi   = i / (ncomp * nf);
            const int  cei  = (i / nf) % ncomp;
            const int  mi   = i % nf;
            const int  b    = P.comps[cei];
            const bool rowD = rhsA[Nt + i] != 0.;
            double     r    = 0.;
            if (!rowD)
              {
                const bool    neu = bcs[fi * 3 + b] == 2.;
                const int64_t Fi  = neu ? face_index(P, cell, fi, DIM) : 0;
                for (int qf = 0; qf < nqf; ++qf)
                  {
                    const int    fq  = fi * nqf + qf;
                    const double E0n = W0n[fq];
                    const bool   cellside = (flux == 0) || (flux == 2 && E0n > 0.);
                    const double tb_ = taus[fi * 3 + b];
                    const double cb0 = c0f[b * F * nqf + fq];
                    const double tb0 = tr0[b * F * nqf + fq];
                    double       v;
                    if (b == 0)
                      v = -eps * E0n - tb_ * cb0 + tb_ * tb0;
                    else
                      {
                        const double mu   = (b == 1) ? mun : mup;
                        const double cstr = cellside ? cb0 : tb0;
                        const double sg   = (b == 1) ? -1. : 1.;
                        v = sg * cstr * mu * E0n + U_T * mu * W0n[b * F * nqf + fq] +
                            tb_ * cb0 - tb_ * tb0;
                      }
                    if (neu && !thermo)
                      v += P.face_bc_val[(Fi * 3 + b) * nqf + qf];
                    r += w_f[fq] * xi[qf * nf + mi] * v;
                  }
                r += rhsA[i];
              }
            P.rhs[cell * Nt + i]   = r;
            P.dflag[cell * Nt + i] = rowD ? 1 : 0;
            P.dval[cell * Nt + i]  = gv[i];
          }
        __syncwarp();
      }
  }

  // --------------------------------------------------------- reconstruct
  // Cell update from the trace update: du = Y0 - Y_t dlam for the scalar
  // unknowns, and the flux unknowns from the (linear) flux rows,
  // W_new = P u_new - Q lam_new, i.e. dW = P(u0+du) - W0 - Q(lam0+dlam).
  template <int DIM, int K>
  __global__ void __launch_bounds__(256)
  reconstruct_kernel(const KParams P, const double *__restrict__ dtrace,
                     double *__restrict__ dcell)
  {
    using Dm          = Dims<DIM, K>;
    constexpr int nb  = Dm::nb;
    constexpr int nf  = Dm::nf;
    constexpr int F   = Dm::F;
    constexpr int NCA = Dm::Nc_all;
    extern __shared__ double smem[];
    const int lane  = threadIdx.x & 31;
    const int warp  = threadIdx.x >> 5;
    const int ncomp = P.ncomp;
    const int Ns    = ncomp * nb;
    const int Nt    = F * ncomp * nf;
    // stage the elimination operators P and Q (contiguous in the table block)
    const int nPQ = P.to.minv - P.to.P;
    for (int i = threadIdx.x; i < nPQ; i += blockDim.x)
      smem[i] = P.tables[P.to.P + i];
    __syncthreads();
    const double *Pm  = smem;
    const double *Qm  = smem + (P.to.Q - P.to.P);
    const int     wsz = Ns + 2 * F * 3 * nf + nb;
    double *ws   = smem + ((nPQ + 1) & ~1) + warp * ((wsz + 1) & ~1);
    double *du   = ws;
    double *dl   = ws + Ns;          // [F][3][nf] trace update
    double *lnew = dl + F * 3 * nf;  // [F][3][nf] lam0 + dlam
    double *unew = lnew + F * 3 * nf;

    for (int64_t cell = (int64_t)blockIdx.x * P.wpb + warp; cell < P.ncells;
         cell += (int64_t)gridDim.x * P.wpb)
      {
        for (int i = lane; i < F * 3 * nf; i += 32)
          {
            const int     f  = i / (3 * nf);
            const int64_t Fi = face_index(P, cell, f, DIM);
            const double  d  = dtrace[Fi * 3 * nf + (i % (3 * nf))];
            dl[i]            = d;
            lnew[i]          = P.trace_state[Fi * 3 * nf + (i % (3 * nf))] + d;
          }
        __syncwarp();
        const double *Y = P.ycache + cell * (int64_t)Ns * P.ycols;
        for (int i = lane; i < Ns; i += 32)
          {
            double v = Y[i];
            for (int t = 0; t < Nt; ++t)
              {
                const int f  = t / (ncomp * nf);
                const int ce = (t / nf) % ncomp;
                const int m  = t % nf;
                v -= Y[(1 + t) * Ns + i] * dl[(f * 3 + P.comps[ce]) * nf + m];
              }
            du[i] = v;
          }
        __syncwarp();
        const double *cs  = P.cell_state + cell * NCA;
        double       *out = dcell + cell * NCA;
        for (int b = 0; b < 3; ++b)
          {
            int ce = -1;
            for (int c = 0; c < ncomp; ++c)
              if (P.comps[c] == b)
                ce = c;
            double *ob = out + b * (DIM + 1) * nb;
            if (ce < 0)
              {
                for (int i = lane; i < (DIM + 1) * nb; i += 32)
                  ob[i] = 0.;
                continue;
              }
            for (int i = lane; i < nb; i += 32)
              {
                ob[DIM * nb + i] = du[ce * nb + i];
                unew[i]          = cs[(b * (DIM + 1) + DIM) * nb + i] + du[ce * nb + i];
              }
            __syncwarp();
            for (int i = lane; i < DIM * nb; i += 32)
              {
                double v = -cs[b * (DIM + 1) * nb + i];
                for (int e = 0; e < nb; ++e)
                  v += Pm[i * nb + e] * unew[e];
                for (int t = 0; t < F * nf; ++t)
                  v -= Qm[i * (F * nf) + t] * lnew[((t / nf) * 3 + b) * nf + (t % nf)];
                ob[i] = v;
              }
            __syncwarp();
          }
      }
  }
} // namespace ddhdg
