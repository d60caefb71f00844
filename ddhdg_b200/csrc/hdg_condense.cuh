// Per-cell assembly + static condensation kernel (sm_100a, FP64).
//
// One CTA of CondenseTPB threads works on one cell at a time (persistent grid,
// stride loop over cells).  The reference's local system
// (include/assembling_methods.template.h:269-2160) is restated in block form:
// the flux unknowns (E, Wn, Wp) are eliminated through the constant mass
// matrix, leaving for the scalar unknowns (V, n, p) of the enabled components
//     S y = R,   R = [residual | ct columns (| drift columns)].
// Every block of S and R is a contraction over "channels" (cell quadrature
// points, their gradient directions, face quadrature points) of per-cell
// coefficients with constant tables staged in shared memory:
//     S_{b b'}[a][e] = sum_ch coef_{b b'}(ch) TL[ch][a] RT[ch][e].
// The coupling coefficients per channel are (test component b, trial b'):
//     alpha  value x value      (plain V-n/p coupling, Boltzmann term, dR/dn)
//     beta   grad x value       (drift of the trial density with E0)
//     kappa  grad x flux        (permittivity, drift with dE, diffusion)
//     gamma  face value x value (stabilisation tau, upwinded drift)
//     rho    face value x flux  (normal flux terms)
// S is row-equilibrated and LU-factorised with partial pivoting; the condensed
// trace system tt + tc cc^-1 [ct | rhs] (T:2651-2686) is evaluated from the
// solved columns as face integrals.  The solved columns stay in HBM for the
// reconstruction.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "hdg_kernels.cuh"

namespace ddhdg
{
  constexpr int CondenseTPB = 128;

  struct Ws2Off
  {
    int coef, lam, c0, W0, qc, c0f, W0n, tr0, Wrc, Wrf, tau, bcs;
    int al, be, ka, ga, rh;             // per pair (9) coefficients
    int ctc, ctd, tcS, tcW, ttc, rhsf;  // per component / pair face data
    int r0, r1, rf;                     // residual coefficients
    int S, R, g, dfl, rhsA, total;
  };

  __host__ __device__ inline Ws2Off
  ws2_layout(int dim, int nb, int nf, int ncomp, int ncol, bool r_global = false)
  {
    const int F = 2 * dim, nqc = nb, Fq = F * nf;
    const int Ns = ncomp * nb, Nt = F * ncomp * nf;
    Ws2Off    o;
    int       p = 0;
    auto      take = [&p](int n) {
      const int r = p;
      p += (n + 1) & ~1;
      return r;
    };
    o.coef  = take(3 * (dim + 1) * nb);
    o.lam   = take(F * 3 * nf);
    o.c0    = take(3 * nqc);
    o.W0    = take(3 * dim * nqc);
    o.qc    = take(6 * nqc);
    o.c0f   = take(3 * Fq);
    o.W0n   = take(3 * Fq);
    o.tr0   = take(3 * Fq);
    o.Wrc   = take(3 * dim * nqc);
    o.Wrf   = take(3 * Fq);
    o.tau   = take(F * 3);
    o.bcs   = take(F * 3);
    o.al    = take(9 * nqc);
    o.be    = take(9 * nqc * dim);
    o.ka    = take(9 * nqc);
    o.ga    = take(9 * Fq);
    o.rh    = take(9 * Fq);
    o.ctc   = take(3 * Fq);
    o.ctd   = take(3 * Fq);
    o.tcS   = take(3 * Fq);
    o.tcW   = take(9 * Fq);
    o.ttc   = take(3 * Fq);
    o.rhsf  = take(3 * Fq);
    o.r0    = take(3 * nqc);
    o.r1    = take(3 * nqc * dim);
    o.rf    = take(3 * Fq);
    o.S     = take(Ns * (Ns + 1));
    o.R     = r_global ? 0 : take(Ns * ncol); // else a slice of KParams::rscratch
    o.g     = take(Nt);
    o.dfl   = take(Nt);
    o.rhsA  = take(Nt);
    o.total = p;
    return o;
  }

  // D += A B for one 8x8x4 FP64 tile on the tensor path (mma.sync m8n8k4):
  // lane l holds A[l/4][l%4], B[l%4][l/4] and D[l/4][2(l%4) + {0,1}]
  __device__ __forceinline__ void
  cta_dmma8x8x4(double &d0, double &d1, double a, double b)
  {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
  }

  constexpr int CtaLuNB = 8; // panel width of the blocked LU

  // The solve of the CTA-per-cell condensation: LU with partial pivoting of
  // the row-equilibrated S (Ns x Ns, row stride ldS) applied to R (Ns x ncol,
  // row stride ncol), then U Y = R' by block back substitution; R becomes Y.
  // Right-looking, panels of CtaLuNB columns:
  // - warp 0 factorises the panel with its rows in registers (pivot search
  //   by one redux of a packed key over the rows below the diagonal, as in
  //   the warp-per-cell Gauss-Jordan; the pivot row exchanged and broadcast
  //   by shuffles; multipliers inside the panel);
  // - the CTA, a thread per column, applies the panel's row swaps to the
  //   columns right of it (S, then R) and solves the panel rows of U there
  //   with the unit lower panel block;
  // - the trailing update A22 -= L21 U12 runs on the FP64 tensor path in
  //   8 x 8 tiles (K = the panel width), the warps taking tiles in turn.
  // Each panel sees its columns fully updated, so the pivots are those of
  // the unblocked factorisation up to the key's rounding (2^-13).  The
  // multipliers of finished panels are not
  // swapped (nothing reads them again).  Back substitution per panel block
  // from the bottom: the diagonal block a thread per column of R, then the
  // rows above on the tensor path.  Three barriers per panel and two per
  // block, against three and two per column unblocked.  Sets sh_sing when a
  // pivot is zero or not finite.
  // NSMAX: the largest Ns (rows of the panel held per lane: NSMAX / 32,
  // rounded up)
  template <int T, int NSMAX>
  __device__ void
  cta_lu_solve(double *S, int ldS, double *R, int ncol, int Ns, int *sh_p, int &sh_sing)
  {
    constexpr int PR = (NSMAX + 31) / 32;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int NW = T / 32;
    const int g = lane >> 2, q = lane & 3;
    for (int j0 = 0; j0 < Ns; j0 += CtaLuNB)
      {
        const int w = min(CtaLuNB, Ns - j0);
        // ---- panel: warp 0, its rows in registers (lane l holds rows
        // j0 + l + 32 r), pivot rows exchanged and broadcast by shuffles
        if (warp == 0)
          {
            double v[PR][CtaLuNB];
#pragma unroll
            for (int r = 0; r < PR; ++r)
              {
                const int row = j0 + lane + 32 * r;
#pragma unroll
                for (int c = 0; c < CtaLuNB; ++c)
                  v[r][c] = (row < Ns && c < w) ? S[row * ldS + j0 + c] : 0.;
              }
#pragma unroll
            for (int jj = 0; jj < CtaLuNB; ++jj)
              {
                if (jj >= w)
                  break;
                const int j    = j0 + jj;
                double    best = -1.;
                int       bi   = Ns;
#pragma unroll
                for (int r = 0; r < PR; ++r)
                  {
                    const int row = j0 + lane + 32 * r;
                    if (row >= j && row < Ns && fabs(v[r][jj]) > best)
                      {
                        best = fabs(v[r][jj]);
                        bi   = row;
                      }
                  }
                // one warp max-reduction of a 32-bit key: the high word of
                // |candidate| with the low 7 bits replaced by 127 - its row
                // offset in the panel (the pivot is within 2^-13 of the
                // largest candidate, ties go to the lowest row)
                unsigned key = 0u;
                if (bi < Ns)
                  key = ((unsigned)((unsigned long long)__double_as_longlong(best) >> 32) & ~127u) |
                        (127u - (unsigned)(bi - j0));
                const unsigned kmax = __reduce_max_sync(0xffffffffu, key);
                bi = kmax ? j0 + 127 - (int)(kmax & 127u) : j; // none: keep the row (singular)
                if (lane == 0)
                  sh_p[jj] = bi;
                const int oj = (j - j0) & 31, sj = (j - j0) >> 5;
                if (bi != j)
                  {
                    const int op = (bi - j0) & 31, sp = (bi - j0) >> 5;
#pragma unroll
                    for (int c = 0; c < CtaLuNB; ++c)
                      {
                        double xp = 0., xj = 0.;
#pragma unroll
                        for (int r = 0; r < PR; ++r)
                          {
                            xp = (r == sp) ? v[r][c] : xp;
                            xj = (r == sj) ? v[r][c] : xj;
                          }
                        xp = __shfl_sync(0xffffffffu, xp, op);
                        xj = __shfl_sync(0xffffffffu, xj, oj);
#pragma unroll
                        for (int r = 0; r < PR; ++r)
                          {
                            if (lane == oj && r == sj)
                              v[r][c] = xp;
                            if (lane == op && r == sp)
                              v[r][c] = xj;
                          }
                      }
                  }
                double prow[CtaLuNB];
#pragma unroll
                for (int c = 0; c < CtaLuNB; ++c)
                  {
                    double x = 0.;
#pragma unroll
                    for (int r = 0; r < PR; ++r)
                      x = (r == sj) ? v[r][c] : x;
                    prow[c] = __shfl_sync(0xffffffffu, x, oj);
                  }
                const double d   = prow[jj];
                const double inv = (d != 0.) ? 1. / d : 0.;
                if (lane == 0 && (!(fabs(d) > 0.) || !isfinite(d)))
                  sh_sing = 1;
#pragma unroll
                for (int r = 0; r < PR; ++r)
                  {
                    const int row = j0 + lane + 32 * r;
                    if (row > j && row < Ns)
                      {
                        const double l = v[r][jj] * inv;
                        v[r][jj]       = l;
#pragma unroll
                        for (int c = jj + 1; c < CtaLuNB; ++c)
                          if (c < w)
                            v[r][c] -= l * prow[c];
                      }
                  }
              }
#pragma unroll
            for (int r = 0; r < PR; ++r)
              {
                const int row = j0 + lane + 32 * r;
                if (row < Ns)
#pragma unroll
                  for (int c = 0; c < CtaLuNB; ++c)
                    if (c < w)
                      S[row * ldS + j0 + c] = v[r][c];
              }
          }
        __syncthreads();
        // ---- swaps and U12 on the columns right of the panel: S, then R
        const int nSr = Ns - j0 - w;
        for (int v = tid; v < nSr + ncol; v += T)
          {
            double   *col = (v < nSr) ? S + j0 + w + v : R + (v - nSr);
            const int ld  = (v < nSr) ? ldS : ncol;
            double    x[CtaLuNB];
#pragma unroll
            for (int jj = 0; jj < CtaLuNB; ++jj)
              if (jj < w)
                {
                  const int p = sh_p[jj], j = j0 + jj;
                  if (p != j)
                    {
                      const double t0 = col[j * ld];
                      col[j * ld]     = col[p * ld];
                      col[p * ld]     = t0;
                    }
                }
#pragma unroll
            for (int jj = 0; jj < CtaLuNB; ++jj)
              if (jj < w)
                {
                  double y = col[(j0 + jj) * ld];
#pragma unroll
                  for (int t = 0; t < CtaLuNB; ++t)
                    if (t < jj)
                      y -= S[(j0 + jj) * ldS + j0 + t] * x[t];
                  x[jj] = y;
                }
#pragma unroll
            for (int jj = 0; jj < CtaLuNB; ++jj)
              if (jj < w)
                col[(j0 + jj) * ld] = x[jj];
          }
        __syncthreads();
        // ---- trailing update A22 -= L21 U12 (8 x 8 tiles on the tensor path)
        const int r0 = j0 + w, nr = Ns - r0;
        if (nr > 0)
          {
            const int nrt = (nr + 7) / 8, nct = (nSr + ncol + 7) / 8;
            for (int tile = warp; tile < nrt * nct; tile += NW)
              {
                const int rt = tile % nrt, ct = tile / nrt;
                const int row = r0 + rt * 8 + g;  // A-fragment row, D row
                const int vb  = ct * 8 + g;       // B-fragment column
                double    d0 = 0., d1 = 0.;
#pragma unroll
                for (int ks = 0; ks < CtaLuNB; ks += 4)
                  {
                    const int    k = ks + q;
                    const double a = (k < w && row < Ns) ? S[row * ldS + j0 + k] : 0.;
                    double       b = 0.;
                    if (k < w && vb < nSr + ncol)
                      b = (vb < nSr) ? S[(j0 + k) * ldS + r0 + vb] : R[(j0 + k) * ncol + vb - nSr];
                    cta_dmma8x8x4(d0, d1, a, b);
                  }
                if (row < Ns)
                  {
#pragma unroll
                    for (int e = 0; e < 2; ++e)
                      {
                        const int    v  = ct * 8 + 2 * q + e;
                        const double dv = e ? d1 : d0;
                        if (v < nSr)
                          S[row * ldS + r0 + v] -= dv;
                        else if (v < nSr + ncol)
                          R[row * ncol + v - nSr] -= dv;
                      }
                  }
              }
          }
        __syncthreads();
      }
    // ---- back substitution U Y = R', blocks of the panels from the bottom
    const int last = (Ns - 1) / CtaLuNB * CtaLuNB;
    for (int j0 = last; j0 >= 0; j0 -= CtaLuNB)
      {
        const int w = min(CtaLuNB, Ns - j0);
        for (int c = tid; c < ncol; c += T)
          {
            double y[CtaLuNB];
#pragma unroll
            for (int jj = CtaLuNB - 1; jj >= 0; --jj)
              if (jj < w)
                {
                  double acc = R[(j0 + jj) * ncol + c];
#pragma unroll
                  for (int t = 0; t < CtaLuNB; ++t)
                    if (t > jj && t < w)
                      acc -= S[(j0 + jj) * ldS + j0 + t] * y[t];
                  const double d = S[(j0 + jj) * ldS + j0 + jj];
                  y[jj]          = acc * ((d != 0.) ? 1. / d : 0.);
                }
#pragma unroll
            for (int jj = 0; jj < CtaLuNB; ++jj)
              if (jj < w)
                R[(j0 + jj) * ncol + c] = y[jj];
          }
        __syncthreads();
        if (j0 > 0)
          {
            const int nrt = (j0 + 7) / 8, nct = (ncol + 7) / 8;
            for (int tile = warp; tile < nrt * nct; tile += NW)
              {
                const int rt = tile % nrt, ct = tile / nrt;
                const int row = rt * 8 + g, cb = ct * 8 + g;
                double    d0 = 0., d1 = 0.;
#pragma unroll
                for (int ks = 0; ks < CtaLuNB; ks += 4)
                  {
                    const int    k = ks + q;
                    const double a = (k < w && row < j0) ? S[row * ldS + j0 + k] : 0.;
                    const double b = (k < w && cb < ncol) ? R[(j0 + k) * ncol + cb] : 0.;
                    cta_dmma8x8x4(d0, d1, a, b);
                  }
                if (row < j0)
                  {
#pragma unroll
                    for (int e = 0; e < 2; ++e)
                      {
                        const int c = ct * 8 + 2 * q + e;
                        if (c < ncol)
                          R[row * ncol + c] -= e ? d1 : d0;
                      }
                  }
              }
            __syncthreads();
          }
      }
  }

  // The body of the CTA-per-cell condensation: the CTA (T threads, a
  // multiple of 32: CondenseTPB in condense2_kernel, fewer in the batched
  // launch) works through the cells cell_begin, cell_begin + cell_step, ...
  // < cell_end with the workspace at smem (tables first when P.stage) and,
  // for R outside shared memory, the R slice `slot` of P.rscratch.
  template <int DIM, int K, int T = CondenseTPB>
  __device__ __forceinline__ void
  condense2_cells(const KParams &P, double *smem, int64_t slot, int64_t cell_begin,
                  int64_t cell_end, int64_t cell_step)
  {
    using Dm          = Dims<DIM, K>;
    constexpr int nb  = Dm::nb;
    constexpr int nf  = Dm::nf;
    constexpr int nqc = Dm::nqc;
    constexpr int nqf = Dm::nqf;
    constexpr int F   = Dm::F;
    constexpr int Fq  = F * nqf;
    constexpr int Ft  = F * nf;
    constexpr int NCA = Dm::Nc_all;
    constexpr int NW  = T / 32;
    __shared__ int sh_p8[CtaLuNB];
    __shared__ int sh_sing;

    const int tid   = threadIdx.x;
    const int lane  = tid & 31;
    const int warp  = tid >> 5;
    const int ncomp = P.ncomp;
    const int Ns    = ncomp * nb;
    const int Nt    = F * ncomp * nf;
    const int ncol  = P.ncol;
    const int ldS   = Ns + 1;
    const bool two  = ncol > 1 + Nt;

    // ---- constant tables, staged once per CTA
    const double *tb = P.tables;
    if (P.stage)
      {
        for (int i = tid; i < P.to.total; i += T)
          smem[i] = P.tables[i];
        __syncthreads();
        tb = smem;
      }
    const double *phi_c  = tb + P.to.phi_c;
    const double *w_f    = tb + P.to.w_f;
    const double *xi     = tb + P.to.xi;
    const double *fminvw = tb + P.to.fminvw;
    const double *phi_f  = tb + P.to.phi_f; // = RTg  [fq][nb]
    const double *TLc    = tb + P.to.TLc;
    const double *TLg    = tb + P.to.TLg;
    const double *TLf    = tb + P.to.TLf;
    const double *RTk    = tb + P.to.RTk;
    const double *RTr    = tb + P.to.RTr;
    const double *RQk    = tb + P.to.RQk;
    const double *RQr    = tb + P.to.RQr;
    const double *PW_c   = tb + P.to.PW_c;
    const double *PW_f   = tb + P.to.PW_f;
    const double *QW_c   = tb + P.to.QW_c;
    const double *QW_f   = tb + P.to.QW_f;

    const Ws2Off wo = ws2_layout(DIM, nb, nf, ncomp, ncol, P.rscratch != nullptr);
    double *ws = smem + (P.stage ? ((P.to.total + 1) & ~1) : 0);
    double *coef = ws + wo.coef, *lam = ws + wo.lam, *c0 = ws + wo.c0, *W0 = ws + wo.W0,
           *qc = ws + wo.qc, *c0f = ws + wo.c0f, *W0n = ws + wo.W0n, *tr0 = ws + wo.tr0,
           *Wrc = ws + wo.Wrc, *Wrf = ws + wo.Wrf, *taus = ws + wo.tau, *bcs = ws + wo.bcs,
           *al = ws + wo.al, *be = ws + wo.be, *ka = ws + wo.ka, *ga = ws + wo.ga,
           *rh = ws + wo.rh, *ctc = ws + wo.ctc, *ctd = ws + wo.ctd, *tcS = ws + wo.tcS,
           *tcW = ws + wo.tcW, *ttc = ws + wo.ttc, *rhsf = ws + wo.rhsf, *r0 = ws + wo.r0,
           *r1 = ws + wo.r1, *rf = ws + wo.rf, *S = ws + wo.S, *R = ws + wo.R,
           *gv = ws + wo.g, *dfl = ws + wo.dfl, *rhsA = ws + wo.rhsA;
    // R of the largest systems (3D k = 2 with drift columns: 210 KB) lives
    // in this CTA's slice of a global buffer, which stays in L2
    if (P.rscratch)
      R = P.rscratch + slot * Ns * ncol;

    const double eps = P.eps, mun = P.mun, mup = P.mup, U_T = P.U_T;
    const bool   thermo   = P.thermo != 0;
    const bool   phi_mode = thermo || P.phi_linearize;
    const double ds       = (P.jfix & 1) ? -1. : 1.;
    const int    flux     = P.flux;
    int          ce_of[3] = {-1, -1, -1};
    for (int c = 0; c < ncomp; ++c)
      ce_of[P.comps[c]] = c;
    const bool nen = ce_of[1] >= 0, pen = ce_of[2] >= 0;

    for (int64_t cell = cell_begin; cell < cell_end; cell += cell_step)
      {
        // ------------------------------------------------------ state
        const double *cs = P.cell_state + cell * NCA;
        for (int i = tid; i < NCA; i += T)
          coef[i] = cs[i];
        for (int i = tid; i < F * 3 * nf; i += T)
          {
            const int64_t Fi = face_index(P, cell, i / (3 * nf), DIM);
            lam[i]           = P.trace_state[Fi * 3 * nf + (i % (3 * nf))];
          }
        for (int i = tid; i < F * 3; i += T)
          {
            const int     f  = i / 3, b = i % 3;
            const int64_t Fi = face_index(P, cell, f, DIM);
            taus[i] = P.tau_table ? P.tau_table[(cell * F + f) * 3 + b] : P.tau[b];
            bcs[i]  = (double)P.face_bc[Fi * 3 + b];
          }
        __syncthreads();

        // ------------------------------------- fields at quadrature points
        for (int i = tid; i < 3 * (DIM + 1) * nqc; i += T)
          {
            const int     b  = i / ((DIM + 1) * nqc);
            const int     s  = (i / nqc) % (DIM + 1);
            const int     q  = i % nqc;
            const double *cf = coef + (b * (DIM + 1) + s) * nb;
            double        v  = 0.;
#pragma unroll
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
            const int     f  = fq / nqf, qf = fq % nqf;
            const int     ax = f / 2;
            const double  sg = (f & 1) ? 1. : -1.;
            const double *ph = phi_f + fq * nb;
            const double *cS = coef + (b * (DIM + 1) + DIM) * nb;
            const double *cW = coef + (b * (DIM + 1) + ax) * nb;
            double        u = 0., wn = 0., t = 0.;
#pragma unroll
            for (int a = 0; a < nb; ++a)
              {
                u += ph[a] * cS[a];
                wn += ph[a] * cW[a];
              }
#pragma unroll
            for (int m = 0; m < nf; ++m)
              t += xi[qf * nf + m] * lam[(f * 3 + b) * nf + m];
            c0f[i] = u;
            W0n[i] = sg * wn;
            tr0[i] = t;
          }
        __syncthreads();

        // ---------------- point coefficients and the flux residual field
        for (int q = tid; q < nqc; q += T)
          {
            const double n0 = c0[nqc + q], p0 = c0[2 * nqc + q], V0 = c0[q];
            double       r = 0., drn = 0., drp = 0.;
            if (nen || pen)
              {
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
                const double KbT = KB_ * P.T / (Q_ * P.V_rescale);
                const double evr = P.ev / (Q_ * P.V_rescale);
                const double ecr = P.ec / (Q_ * P.V_rescale);
                double       phn = 0., php = 0.;
                if (!thermo)
                  {
                    // quasi Fermi potentials (include/solver.h:343-376)
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
            qc[5 * nqc + q] = P.doping[cell * nqc + q];
          }
        // flux residual W = P u0 - W0 - Q lam0 at cell and face points
        for (int i = tid; i < ncomp * DIM * nqc; i += T)
          {
            const int     ce = i / (DIM * nqc);
            const int     b  = P.comps[ce];
            const int     s  = (i / nqc) % DIM;
            const int     q  = i % nqc;
            const double *cS = coef + (b * (DIM + 1) + DIM) * nb;
            double        v  = -W0[(b * DIM + s) * nqc + q];
#pragma unroll
            for (int e = 0; e < nb; ++e)
              v += PW_c[(e * nqc + q) * DIM + s] * cS[e];
#pragma unroll 4
            for (int t = 0; t < Ft; ++t)
              v -= QW_c[(t * nqc + q) * DIM + s] * lam[((t / nf) * 3 + b) * nf + (t % nf)];
            Wrc[(ce * DIM + s) * nqc + q] = v;
          }
        for (int i = tid; i < ncomp * Fq; i += T)
          {
            const int     ce = i / Fq;
            const int     b  = P.comps[ce];
            const int     fq = i % Fq;
            const int     f = fq / nqf, qf = fq % nqf;
            const double *cS = coef + (b * (DIM + 1) + DIM) * nb;
            double        v  = -W0n[b * Fq + fq];
#pragma unroll
            for (int e = 0; e < nb; ++e)
              v += PW_f[(e * F + f) * nqf + qf] * cS[e];
#pragma unroll 4
            for (int t = 0; t < Ft; ++t)
              v -= QW_f[(t * F + f) * nqf + qf] * lam[((t / nf) * 3 + b) * nf + (t % nf)];
            Wrf[ce * Fq + fq] = v;
          }
        __syncthreads();

        // ------------------------------------ channel coefficients per pair
        for (int i = tid; i < 9 * nqc; i += T)
          {
            const int    pr = i / nqc, q = i % nqc;
            const int    b = pr / 3, bp = pr % 3;
            const double n0 = c0[nqc + q], p0 = c0[2 * nqc + q];
            double       a_ = 0., k_ = 0., bb[DIM];
#pragma unroll
            for (int s = 0; s < DIM; ++s)
              bb[s] = 0.;
            if (b == 0)
              {
                if (bp == 0)
                  {
                    a_ = phi_mode ? -qc[3 * nqc + q] : 0.;
                    k_ = -eps;
                  }
                else if (!phi_mode)
                  a_ = (bp == 1) ? 1. : -1.;
              }
            else
              {
                if (bp == 0)
                  k_ = (b == 1) ? ds * n0 * mun : -ds * p0 * mup;
                else
                  {
                    a_ = (bp == 1) ? -qc[nqc + q] : -qc[2 * nqc + q];
                    if (bp == b)
                      {
                        k_              = U_T * ((b == 1) ? mun : mup);
                        const double sg = (b == 1) ? -mun : mup;
#pragma unroll
                        for (int s = 0; s < DIM; ++s)
                          bb[s] = sg * W0[s * nqc + q];
                      }
                  }
              }
            al[i] = a_;
            ka[i] = k_;
#pragma unroll
            for (int s = 0; s < DIM; ++s)
              be[i * DIM + s] = bb[s];
          }
        for (int i = tid; i < 9 * Fq; i += T)
          {
            const int    pr = i / Fq, fq = i % Fq, f = fq / nqf;
            const int    b = pr / 3, bp = pr % 3;
            const double E0n = W0n[fq];
            const bool   cellside = (flux == 0) || (flux == 2 && E0n > 0.);
            double       g_ = 0., r_ = 0., w_ = 0.;
            if (b == 0)
              {
                if (bp == 0)
                  {
                    g_ = taus[f * 3];
                    r_ = eps;
                    w_ = -eps;
                  }
              }
            else
              {
                const double mu   = (b == 1) ? mun : mup;
                const double sg   = (b == 1) ? 1. : -1.;
                const double cstr = cellside ? c0f[b * Fq + fq] : tr0[b * Fq + fq];
                if (bp == 0)
                  {
                    r_ = sg * mu * cstr;
                    w_ = -sg * mu * cstr;
                  }
                else if (bp == b)
                  {
                    g_ = (cellside ? sg * mu * E0n : 0.) - taus[f * 3 + b];
                    r_ = -U_T * mu;
                    w_ = U_T * mu;
                  }
              }
            ga[i]  = g_;
            rh[i]  = r_;
            tcW[i] = w_;
          }
        for (int i = tid; i < 3 * Fq; i += T)
          {
            const int    b = i / Fq, fq = i % Fq, f = fq / nqf, qf = fq % nqf;
            const double E0n = W0n[fq];
            const bool   cellside = (flux == 0) || (flux == 2 && E0n > 0.);
            const bool   drift    = (flux == 1) || (flux == 2 && E0n <= 0.);
            const double tb_ = taus[f * 3 + b];
            const double cb0 = c0f[b * Fq + fq], tb0 = tr0[b * Fq + fq];
            double       c_, d_ = 0., s_, t_, rr;
            if (b == 0)
              {
                c_ = -tb_;
                s_ = -tb_;
                t_ = -tb_;
                rr = -eps * E0n - tb_ * cb0 + tb_ * tb0;
              }
            else
              {
                const double mu   = (b == 1) ? mun : mup;
                const double sg   = (b == 1) ? 1. : -1.;
                const double cstr = cellside ? cb0 : tb0;
                c_                = tb_;
                d_                = drift ? sg * mu * E0n : 0.;
                s_                = (cellside ? -sg * mu * E0n : 0.) + tb_;
                t_                = tb_ + d_;
                rr = -sg * cstr * mu * E0n + U_T * mu * W0n[b * Fq + fq] + tb_ * cb0 - tb_ * tb0;
              }
            const bool neu = bcs[f * 3 + b] == 2.;
            if (neu && !thermo)
              {
                const int64_t Fi = face_index(P, cell, f, DIM);
                rr += P.face_bc_val[(Fi * 3 + b) * nqf + qf];
              }
            ctc[i]  = c_;
            ctd[i]  = d_;
            tcS[i]  = s_;
            ttc[i]  = t_;
            rhsf[i] = rr;
          }
        __syncthreads();

        // ------------------------------------------ residual coefficients
        for (int i = tid; i < ncomp * nqc; i += T)
          {
            const int    ce = i / nqc, q = i % nqc, b = P.comps[ce];
            const double n0 = c0[nqc + q], p0 = c0[2 * nqc + q];
            double       v0, v1[DIM];
            if (b == 0)
              {
                v0 = qc[5 * nqc + q] + (phi_mode ? qc[4 * nqc + q] : (p0 - n0));
#pragma unroll
                for (int s = 0; s < DIM; ++s)
                  v1[s] = eps * W0[s * nqc + q];
              }
            else
              {
                const double mu = (b == 1) ? mun : mup;
                const double cb = (b == 1) ? n0 : -p0;
                v0              = qc[q];
#pragma unroll
                for (int s = 0; s < DIM; ++s)
                  v1[s] = cb * mu * W0[s * nqc + q] - U_T * mu * W0[(b * DIM + s) * nqc + q];
              }
            for (int cp = 0; cp < ncomp; ++cp)
              {
                const double k_ = ka[(b * 3 + P.comps[cp]) * nqc + q];
#pragma unroll
                for (int s = 0; s < DIM; ++s)
                  v1[s] -= k_ * Wrc[(cp * DIM + s) * nqc + q];
              }
            r0[ce * nqc + q] = v0;
#pragma unroll
            for (int s = 0; s < DIM; ++s)
              r1[(ce * nqc + q) * DIM + s] = v1[s];
          }
        for (int i = tid; i < ncomp * Fq; i += T)
          {
            const int    ce = i / Fq, fq = i % Fq, b = P.comps[ce];
            const double E0n = W0n[fq];
            const bool   cellside = (flux == 0) || (flux == 2 && E0n > 0.);
            const double tb_ = taus[(fq / nqf) * 3 + b];
            const double cb0 = c0f[b * Fq + fq], tb0 = tr0[b * Fq + fq];
            double       v;
            if (b == 0)
              v = tb_ * tb0 - eps * E0n - tb_ * cb0;
            else
              {
                const double mu   = (b == 1) ? mun : mup;
                const double sg   = (b == 1) ? 1. : -1.;
                const double cstr = cellside ? cb0 : tb0;
                const double Jf   = sg * cstr * mu * E0n - U_T * mu * W0n[b * Fq + fq];
                v                 = -tb_ * tb0 - Jf + tb_ * cb0;
              }
            for (int cp = 0; cp < ncomp; ++cp)
              v -= rh[(b * 3 + P.comps[cp]) * Fq + fq] * Wrf[cp * Fq + fq];
            rf[ce * Fq + fq] = v;
          }
        // Dirichlet increments (T:1592-1691)
        for (int t = tid; t < Nt; t += T)
          {
            const int f = t / (ncomp * nf), ce = (t / nf) % ncomp, m = t % nf;
            const int b = P.comps[ce];
            double    g = 0., fl = 0.;
            if (bcs[f * 3 + b] == 1.)
              {
                fl = 1.;
                if (!thermo)
                  {
                    const int64_t Fi = face_index(P, cell, f, DIM);
#pragma unroll
                    for (int qf = 0; qf < nqf; ++qf)
                      g += fminvw[m * nqf + qf] *
                           (P.face_bc_val[(Fi * 3 + b) * nqf + qf] - tr0[(b * F + f) * nqf + qf]);
                  }
              }
            gv[t]  = g;
            dfl[t] = fl;
          }
        __syncthreads();

        // ------------------------------------------------ scalar system S
        for (int idx = tid; idx < ncomp * ncomp * nb * nb; idx += T)
          {
            const int blk = idx / (nb * nb);
            const int r_  = idx % (nb * nb);
            const int a = r_ / nb, e = r_ % nb;
            const int ci = blk / ncomp, cj = blk % ncomp;
            const int pr = P.comps[ci] * 3 + P.comps[cj];
            const double *alp = al + pr * nqc;
            const double *kap = ka + pr * nqc;
            const double *bep = be + pr * nqc * DIM;
            const double *gap = ga + pr * Fq;
            const double *rhp = rh + pr * Fq;
            double        v   = 0.;
#pragma unroll
            for (int q = 0; q < nqc; ++q)
              {
                const double pe = phi_c[q * nb + e];
                double       lt = alp[q] * TLc[q * nb + a];
#pragma unroll
                for (int s = 0; s < DIM; ++s)
                  {
                    const double tg = TLg[(q * DIM + s) * nb + a];
                    lt += bep[q * DIM + s] * tg;
                    v += kap[q] * tg * RTk[(q * DIM + s) * nb + e];
                  }
                v += lt * pe;
              }
#pragma unroll
            for (int fq = 0; fq < Fq; ++fq)
              v += TLf[fq * nb + a] * (gap[fq] * phi_f[fq * nb + e] + rhp[fq] * RTr[fq * nb + e]);
            S[(ci * nb + a) * ldS + cj * nb + e] = v;
          }

        // --------------------------------------------------------- R
        // column 0: residual
        for (int i = tid; i < Ns; i += T)
          {
            const int     ce = i / nb, a = i % nb;
            const double *r0p = r0 + ce * nqc;
            const double *r1p = r1 + ce * nqc * DIM;
            const double *rfp = rf + ce * Fq;
            double        v   = 0.;
#pragma unroll
            for (int q = 0; q < nqc; ++q)
              {
                v += TLc[q * nb + a] * r0p[q];
#pragma unroll
                for (int s = 0; s < DIM; ++s)
                  v += TLg[(q * DIM + s) * nb + a] * r1p[q * DIM + s];
              }
#pragma unroll
            for (int fq = 0; fq < Fq; ++fq)
              v += TLf[fq * nb + a] * rfp[fq];
            R[i * ncol] = v;
          }
        // trace columns: ct_z - A_zW Q  (and the drift parts)
        for (int idx = tid; idx < Ns * Nt; idx += T)
          {
            const int i = idx / Nt, t = idx % Nt;
            const int ci = i / nb, a = i % nb;
            const int ft = t / (ncomp * nf), ct = (t / nf) % ncomp, mt = t % nf;
            const int pr = P.comps[ci] * 3 + P.comps[ct];
            const int tq = ft * nf + mt;
            const double *kap = ka + pr * nqc;
            const double *rhp = rh + pr * Fq;
            double        v   = 0., vd = 0.;
#pragma unroll
            for (int q = 0; q < nqc; ++q)
              {
                double gk = 0.;
#pragma unroll
                for (int s = 0; s < DIM; ++s)
                  gk += TLg[(q * DIM + s) * nb + a] * RQk[(q * DIM + s) * Ft + tq];
                v -= kap[q] * gk;
              }
#pragma unroll
            for (int fq = 0; fq < Fq; ++fq)
              v -= rhp[fq] * TLf[fq * nb + a] * RQr[fq * Ft + tq];
            if (ci == ct)
              {
                const int b = P.comps[ci];
#pragma unroll
                for (int qf = 0; qf < nqf; ++qf)
                  {
                    const int    fq = ft * nqf + qf;
                    const double tx = TLf[fq * nb + a] * xi[qf * nf + mt];
                    v += ctc[b * Fq + fq] * tx;
                    vd += ctd[b * Fq + fq] * tx;
                  }
              }
            R[i * ncol + 1 + t] = v;
            if (two)
              R[i * ncol + 1 + Nt + t] = vd;
          }
        if (tid == 0)
          sh_sing = 0;
        __syncthreads();

        // -------------------------- equilibrate rows, LU with partial pivoting
        for (int i = warp; i < Ns; i += NW)
          {
            double mx = 0.;
            for (int j = lane; j < Ns; j += 32)
              mx = fmax(mx, fabs(S[i * ldS + j]));
#pragma unroll
            for (int o = 16; o > 0; o >>= 1)
              mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
            const double sc = (mx > 0.) ? 1. / mx : 1.;
            for (int j = lane; j < Ns; j += 32)
              S[i * ldS + j] *= sc;
            for (int c = lane; c < ncol; c += 32)
              R[i * ncol + c] *= sc;
          }
        __syncthreads();
        cta_lu_solve<T, 3 * nb>(S, ldS, R, ncol, Ns, sh_p8, sh_sing);
        if (tid == 0 && sh_sing)
          atomicExch(P.status, 3);

        // ------------------------ keep Y for the reconstruction [col][row]
        {
          double *yc = P.ycache + cell * (int64_t)Ns * P.ycols;
          for (int idx = tid; idx < Ns * P.ycols; idx += T)
            yc[idx] = R[(idx % Ns) * ncol + idx / Ns];
        }

        // ---- tt = T Y + tc_W Q_t + face block, and the rows' rhs parts, on
        // the FP64 tensor path.  T = tc_c + tc_W P (Nt x Ns: the trace rows'
        // face integrals of the scalar values and normal fluxes) is formed
        // on the fly as the A fragments; a warp takes 8 trace rows at a time
        // against all 1 + Nt columns of Y (the residual column, then the
        // trace columns with their drift columns added), and the epilogue
        // adds the direct face terms: tc_W times the flux's own dependence
        // on the residual (column 0) or on the trace (RQr), and the face
        // block of tt.  The row's right-hand side part is the residual
        // column minus the Dirichlet columns times their values, summed over
        // the four lanes that hold the row.
        {
          constexpr int NTM    = F * 3 * nf;        // trace columns at most
          constexpr int NNT    = (NTM + 8) / 8;     // column tiles of 1 + Nt columns
          const int     g      = lane >> 2, tq = lane & 3;
          double       *tt_out = P.tt + cell * (int64_t)Nt * Nt;
          for (int m0 = warp * 8; m0 < Nt; m0 += NW * 8)
            {
              const int  i   = m0 + g;
              const bool iok = i < Nt;
              const int  ii  = iok ? i : 0;
              const int  fi = ii / (ncomp * nf), ci = (ii / nf) % ncomp, mi = ii % nf;
              const int  b  = P.comps[ci];
              double     wrow[nqf];
#pragma unroll
              for (int qf = 0; qf < nqf; ++qf)
                wrow[qf] = w_f[fi * nqf + qf] * xi[qf * nf + mi];
              double d[NNT][2];
#pragma unroll
              for (int nt = 0; nt < NNT; ++nt)
                d[nt][0] = d[nt][1] = 0.;
              for (int k0 = 0; k0 < Ns; k0 += 4)
                {
                  const int j  = k0 + tq;
                  double    av = 0.;
                  if (iok && j < Ns)
                    {
                      const int     cj = j / nb, e = j % nb;
                      const double *tw = tcW + (b * 3 + P.comps[cj]) * Fq + fi * nqf;
                      const double *ts = tcS + b * Fq + fi * nqf;
                      const bool    sc = cj == ci;
#pragma unroll
                      for (int qf = 0; qf < nqf; ++qf)
                        {
                          const int fq = fi * nqf + qf;
                          av += wrow[qf] * (tw[qf] * RTr[fq * nb + e] + (sc ? ts[qf] * phi_f[fq * nb + e] : 0.));
                        }
                    }
#pragma unroll
                  for (int nt = 0; nt < NNT; ++nt)
                    {
                      const int col = nt * 8 + g; // B-fragment column
                      double    bv  = 0.;
                      if (j < Ns && col < 1 + Nt)
                        {
                          bv = R[j * ncol + col];
                          if (two && col > 0)
                            bv += R[j * ncol + col + Nt];
                        }
                      cta_dmma8x8x4(d[nt][0], d[nt][1], av, bv);
                    }
                }
              const bool rok   = iok && dfl[ii] == 0.;
              double     rpart = 0.;
#pragma unroll
              for (int nt = 0; nt < NNT; ++nt)
#pragma unroll
                for (int e = 0; e < 2; ++e)
                  {
                    const int col = nt * 8 + 2 * tq + e;
                    if (!iok || col >= 1 + Nt)
                      continue;
                    double x = d[nt][e];
                    if (col == 0)
                      {
#pragma unroll
                        for (int qf = 0; qf < nqf; ++qf)
                          for (int cp = 0; cp < ncomp; ++cp)
                            x += wrow[qf] * tcW[(b * 3 + P.comps[cp]) * Fq + fi * nqf + qf] *
                                 Wrf[cp * Fq + fi * nqf + qf];
                        rpart += x;
                        continue;
                      }
                    const int t  = col - 1;
                    const int ft = t / (ncomp * nf), ct = (t / nf) % ncomp, mt = t % nf;
                    const double *tw = tcW + (b * 3 + P.comps[ct]) * Fq + fi * nqf;
#pragma unroll
                    for (int qf = 0; qf < nqf; ++qf)
                      x += wrow[qf] * tw[qf] * RQr[(fi * nqf + qf) * Ft + ft * nf + mt];
                    const bool cD = dfl[t] != 0.;
                    if (cD)
                      rpart -= x * gv[t];
                    double o = 0.;
                    if (rok && !cD)
                      {
                        o = x;
                        if (ft == fi && ct == ci)
#pragma unroll
                          for (int qf = 0; qf < nqf; ++qf)
                            o += wrow[qf] * ttc[b * Fq + fi * nqf + qf] * xi[qf * nf + mt];
                      }
                    tt_out[(int64_t)i * Nt + t] = o;
                  }
              rpart += __shfl_xor_sync(0xffffffffu, rpart, 1);
              rpart += __shfl_xor_sync(0xffffffffu, rpart, 2);
              if (iok && tq == 0)
                rhsA[i] = rpart;
            }
        }
        __syncthreads();

        // ------------------------------------- right-hand side and flags
        for (int i = tid; i < Nt; i += T)
          {
            const int fi = i / (ncomp * nf), ci = (i / nf) % ncomp, mi = i % nf;
            const int b  = P.comps[ci];
            const bool rowD = dfl[i] != 0.;
            double     r    = 0.;
            if (!rowD)
              {
#pragma unroll
                for (int qf = 0; qf < nqf; ++qf)
                  r += w_f[fi * nqf + qf] * xi[qf * nf + mi] * rhsf[b * Fq + fi * nqf + qf];
                r += rhsA[i];
              }
            P.rhs[cell * Nt + i]   = r;
            P.dflag[cell * Nt + i] = rowD ? 1 : 0;
            P.dval[cell * Nt + i]  = gv[i];
          }
        __syncthreads();
      }
  }

  template <int DIM, int K>
  __global__ void __launch_bounds__(CondenseTPB)
  condense2_kernel(const KParams P)
  {
    extern __shared__ double smem[];
    condense2_cells<DIM, K>(P, smem, blockIdx.x, P.cell0 + blockIdx.x, P.ncells, gridDim.x);
  }
} // namespace ddhdg
