// Per-cell assembly + static condensation, one warp per cell (sm_100a), for
// local scalar systems of at most 32 unknowns (3 (k+1)^d <= 32: 1D, 2D
// k <= 2, 3D k = 1), in FP64 or with an FP32 Jacobian (JT = float).
//
// Same mathematics as condense2_kernel (hdg_condense.cuh): the flux unknowns
// are eliminated through the constant mass matrix and the scalar system
// S y = R of the enabled components is solved for the residual and for every
// trace dof.  The execution model differs: every lane owns one row of S in
// registers and the Gauss-Jordan inverse runs as a short loop over the
// columns (virtual partial pivoting with a warp max-reduction of a packed
// pivot key; the register row is rotated by one position per step so that
// the current column is always register 0); Y = S^-1 R and the condensed
// trace matrix tt = T Y + (face terms) are products on the FP64 tensor path
// (mma.sync m8n8k4, 8 x 8 tiles), with the face terms added per output in
// the epilogue.  Warps are independent; the tables used at lane-uniform
// addresses travel in the constant bank (a __grid_constant__ parameter),
// the others are read through the L1 cache.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "hdg_condense.cuh"

namespace ddhdg
{
  constexpr int Condense3MaxWPB = 8; // warps (cells) per CTA at most

  // D += A B for one 8x8x4 FP64 tile on the tensor path (mma.sync m8n8k4):
  // lane l holds A[l/4][l%4], B[l%4][l/4] and D[l/4][2(l%4) + {0,1}]
  __device__ __forceinline__ void
  dmma8x8x4(double &d0, double &d1, double a, double b)
  {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
  }

  // row stride of the staged S^-1 (>= its padded width, = 4 mod 16 doubles:
  // the A-fragment loads of a half warp hit 16 different 8-byte banks)
  __host__ __device__ constexpr int
  sinv_stride(int nsmax)
  {
    int kp = (nsmax + 3) / 4 * 4;
    while (kp % 16 != 4)
      ++kp;
    return kp;
  }

  // Constant tables read at lane-uniform addresses in fully unrolled loops.
  // They travel as a kernel parameter (constant bank), so that the FMAs take
  // them as constant operands; at most 14.4 KB (3D, degree 1).  They are the
  // tables of the unit cell: the elimination operators P = M^-1 G and
  // Q = M^-1 C_W of axis s scale exactly as 1 / h_s, and that factor
  // (KParams::ih) goes into the per-cell coefficient that multiplies them, so
  // that devices of every mesh size share one copy.
  template <int DIM, int K>
  struct CTab
  {
    using Dm                 = Dims<DIM, K>;
    static constexpr int nb  = Dm::nb;
    static constexpr int nqc = Dm::nqc;
    static constexpr int Fq  = Dm::F * Dm::nqf;
    static constexpr int Ft  = Dm::F * Dm::nf;
    double               phi_c[nqc * nb];       // [q][e]
    double               RTk[nqc * DIM * nb];   // [q, s][e]
    double               phi_f[Fq * nb];        // [fq][e]
    double               RTr[Fq * nb];          // [fq][e]
    double               RQk[nqc * DIM * Ft];   // [q, s][t]
    double               RQr[Fq * Ft];          // [fq][t]
    double               xi[Dm::nqf * Dm::nf];  // [qf][m]
  };

  struct Ws3Off
  {
    // dead once Y is formed; the trace-row arrays below overlay them
    int coef, lam, c0, W0, qc, c0f, W0n, tr0, Wrc, tau, bcs;
    int al, be, ka, ga, rh, ctc, ctd, r0, r1, rf;
    // trace-row data of the condensation (overlay)
    int Trs, rA, rS, rD, rZ, H;
    // live to the end of the cell
    int tcS, tcW, ttc, rhsf, Wrf, R, g, dfl, Yc, total;
    int ldr; // row stride of R / Y (even: 16-byte aligned rows)
  };

  // row stride, in elements, of the staged S^-1 for a Jacobian type of jb
  // bytes: FP64 as above; FP32 = 4 mod 32 floats, for the same reason
  __host__ __device__ constexpr int
  sinv_stride_for(int nsmax, int jb)
  {
    if (jb == 8)
      return sinv_stride(nsmax);
    int kp = (nsmax + 3) / 4 * 4;
    while (kp % 32 != 4)
      ++kp;
    return kp;
  }

  // Offsets in doubles.  The Jacobian arrays (coefficients of the linearised
  // operators, S, R / Y, T and the trace-row weights) hold elements of jb
  // bytes: 8 in the FP64 kernel, 4 in the mixed one; everything that carries
  // a residual stays FP64.
  __host__ __device__ inline Ws3Off
  ws3_layout(int dim, int nb, int nf, int ncomp, int ncol, int jb = 8)
  {
    const int F = 2 * dim, nqc = nb, Fq = F * nf, nqf = nf;
    const int Ns = ncomp * nb, Nt = F * ncomp * nf;
    Ws3Off    o;
    int       p = 0;
    auto      take = [&p](int n) {
      const int r = p;
      p += (n + 1) & ~1;
      return r;
    };
    // n Jacobian elements, rounded up to whole 16-byte pairs of doubles
    auto take_j = [&take, jb](int n) { return take((n * jb + 7) / 8); };
    o.coef = take(3 * (dim + 1) * nb);
    o.lam  = take(F * 3 * nf);
    o.c0   = take(3 * nqc);
    o.W0   = take(3 * dim * nqc);
    o.qc   = take(6 * nqc);
    o.c0f  = take(3 * Fq);
    o.W0n  = take(3 * Fq);
    o.tr0  = take(3 * Fq);
    o.Wrc  = take(3 * dim * nqc);
    o.tau  = take(F * 3);
    o.bcs  = take(F * 3);
    o.al   = take_j(9 * nqc);
    o.be   = take_j(9 * nqc * dim);
    o.ka   = take_j(9 * nqc);
    o.ga   = take_j(9 * Fq);
    o.rh   = take_j(9 * Fq);
    o.ctc  = take_j(3 * Fq);
    o.ctd  = take_j(3 * Fq);
    o.r0   = take(3 * nqc);
    o.r1   = take(3 * nqc * dim);
    o.rf   = take(3 * Fq);
    const int dead_end = p;
    p     = 0;
    // 3D FP64: the per-row face weights times coefficients (rA, rS, rD) are
    // recomputed where they are used (shared memory sets the warps per SM;
    // the mixed kernel is issue-bound and keeps them)
    const bool rw = dim == 3 && jb == 8;
    o.Trs = take_j(Ns * Nt);
    o.rA  = take_j(rw ? 0 : Nt * 3 * nqf);
    o.rS  = take_j(rw ? 0 : Nt * nqf);
    o.rD  = take_j(rw ? 0 : Nt * nqf);
    o.rZ  = take(Nt);
    o.H   = take(3 * Fq);
    p     = p > dead_end ? p : dead_end;
    {
      // staged S^-1 of the tensor-path Y = S^-1 R ([rows padded to 8][stride])
      const int sv = ((3 * nb + 7) / 8 * 8 * sinv_stride_for(3 * nb, jb) * jb + 7) / 8;
      p            = p > sv ? p : sv;
      p            = (p + 1) & ~1;
    }
    o.tcS  = take_j(3 * Fq);
    o.tcW  = take_j(9 * Fq);
    o.ttc  = take_j(3 * Fq);
    o.rhsf = take(3 * Fq);
    o.Wrf  = take(3 * Fq);
    // R / Y rows: even in FP64 (16-byte rows); odd in FP32, so that one row
    // per lane walks 32 different banks
    o.ldr  = jb == 8 ? (ncol + 1) & ~1 : (ncol | 1);
    o.R    = take_j(Ns * o.ldr);
    o.g    = take(Nt);
    o.dfl  = take(Nt);
    o.Yc   = take(Ns);
    o.total = p;
    return o;
  }

  // 32-bit pivot key of |x|: the high word of an FP64 value (sign, exponent
  // and 20 mantissa bits), the bits of an FP32 value
  __device__ __forceinline__ unsigned
  pivot_key_bits(double x)
  {
    return (unsigned)((unsigned long long)__double_as_longlong(fabs(x)) >> 32);
  }
  __device__ __forceinline__ unsigned
  pivot_key_bits(float x)
  {
    return __float_as_uint(fabsf(x));
  }
  __device__ __forceinline__ void
  store_pair(double *p, double a, double b)
  {
    *reinterpret_cast<double2 *>(p) = make_double2(a, b);
  }
  __device__ __forceinline__ void
  store_pair(float *p, float a, float b)
  {
    *reinterpret_cast<float2 *>(p) = make_float2(a, b);
  }

  // JT: the Jacobian type.  double: the FP64 kernel.  float: the mixed
  // kernel, where the linearised operators, S and its inverse, R / Y, T and
  // the trace-row weights are FP32 and the products accumulate in FP64 on the
  // tensor path, while the state, every residual and the outputs stay FP64
  // (a Newton loop on these blocks converges to the FP64 solution).
  //
  // The body of the warp-per-cell condensation: one warp works through the
  // cells cell_begin, cell_begin + cell_step, ... < cell_end with its own
  // workspace ws (ws3_layout doubles) and pivot list piv [3 (k+1)^d].  The
  // tables C are the kernel's constant-bank parameter in condense3_kernel
  // and a per-device copy in global memory in the batched launch; the
  // arithmetic is the same, so the results are bitwise the same.
  template <int DIM, int K, typename JT>
  __device__ __forceinline__ void
  condense3_cells(const KParams &P, const CTab<DIM, K> &C, double *ws, int *piv,
                  int64_t cell_begin, int64_t cell_end, int64_t cell_step, const double *rqr = nullptr)
  {
    using Dm            = Dims<DIM, K>;
    constexpr int nb    = Dm::nb;
    constexpr int nf    = Dm::nf;
    constexpr int nqc   = Dm::nqc;
    constexpr int nqf   = Dm::nqf;
    constexpr int F     = Dm::F;
    constexpr int Fq    = F * nqf;
    constexpr int Ft    = F * nf;
    constexpr int NCA   = Dm::Nc_all;
    constexpr int NSMAX = 3 * nb;
    constexpr bool RW   = DIM == 3 && sizeof(JT) == 8; // recompute rA / rS / rD (see ws3_layout)
    static_assert(NSMAX <= 32, "one lane per row of the scalar system");

    const int  lane  = threadIdx.x & 31;
    const int  ncomp = P.ncomp;
    const int  Ns    = ncomp * nb;
    const int  Nt    = F * ncomp * nf;
    const int  ncol  = P.ncol;
    const bool two   = ncol > 1 + Nt;

    const double *tb = P.tables;
    const double *phi_c  = tb + P.to.phi_c;
    const double *w_f    = tb + P.to.w_f;
    const double *xi     = tb + P.to.xi;
    const double *fminvw = tb + P.to.fminvw;
    const double *phi_f  = tb + P.to.phi_f;
    const double *TLc    = tb + P.to.TLc;
    const double *TLg    = tb + P.to.TLg;
    const double *TLf    = tb + P.to.TLf;
    const double *RTr    = tb + P.to.RTr;
    // the face-flux table of the trace rows, read at lane-dependent
    // addresses in the tt epilogue: a per-CTA copy in shared memory when
    // the caller staged one (the same values as the table's)
    const double *RQr    = rqr ? rqr : tb + P.to.RQr;
    const double *PW_c   = tb + P.to.PW_c;
    const double *PW_f   = tb + P.to.PW_f;
    const double *QW_c   = tb + P.to.QW_c;
    const double *QW_f   = tb + P.to.QW_f;

    const Ws3Off wo = ws3_layout(DIM, nb, nf, ncomp, ncol, (int)sizeof(JT));
    const auto   jp = [ws](int off) { return reinterpret_cast<JT *>(ws + off); };
    double *coef = ws + wo.coef, *lam = ws + wo.lam, *c0 = ws + wo.c0, *W0 = ws + wo.W0,
           *qc = ws + wo.qc, *c0f = ws + wo.c0f, *W0n = ws + wo.W0n, *tr0 = ws + wo.tr0,
           *Wrc = ws + wo.Wrc, *Wrf = ws + wo.Wrf, *taus = ws + wo.tau, *bcs = ws + wo.bcs,
           *rhsf = ws + wo.rhsf, *r0 = ws + wo.r0, *r1 = ws + wo.r1, *rf = ws + wo.rf,
           *gv = ws + wo.g, *dfl = ws + wo.dfl, *Yc = ws + wo.Yc;
    JT *al = jp(wo.al), *be = jp(wo.be), *ka = jp(wo.ka), *ga = jp(wo.ga), *rh = jp(wo.rh),
       *ctc = jp(wo.ctc), *ctd = jp(wo.ctd), *tcS = jp(wo.tcS), *tcW = jp(wo.tcW),
       *ttc = jp(wo.ttc), *R = jp(wo.R);
    JT     *Trs = jp(wo.Trs), *rA = jp(wo.rA), *rS = jp(wo.rS), *rD = jp(wo.rD);
    double *rZ = ws + wo.rZ, *Hs = ws + wo.H;
    const int ldr  = wo.ldr;
    const int colC = two ? 1 + Nt : 1; // combined trace columns of Y

    const double eps = P.eps, mun = P.mun, mup = P.mup, U_T = P.U_T;
    const bool   thermo   = P.thermo != 0;
    const bool   phi_mode = thermo || P.phi_linearize;
    const double ds       = (P.jfix & 1) ? -1. : 1.;
    const int    flux     = P.flux;
    // enabled component c -> block index, two bits each (no local memory)
    const int  cpk    = (P.comps[0] & 3) | ((P.comps[1] & 3) << 2) | ((P.comps[2] & 3) << 4);
    const auto cmp_of = [cpk](int c) { return (cpk >> (2 * c)) & 3; };
    bool         nen = false, pen = false;
    for (int c = 0; c < ncomp; ++c)
      {
        nen |= cmp_of(c) == 1;
        pen |= cmp_of(c) == 2;
      }
    for (int64_t cell = cell_begin; cell < cell_end; cell += cell_step)
      {
        // keeps the table loads inside the cell loop (no hoisting of
        // thousands of loop-invariant values into registers)
        asm volatile("" ::: "memory");
        // ------------------------------------------------------------ state
        int64_t face_id[F];
#pragma unroll
        for (int f = 0; f < F; ++f)
          face_id[f] = face_index(P, cell, f, DIM);
        const double *cs = P.cell_state + cell * NCA;
        for (int i = lane; i < NCA; i += 32)
          coef[i] = cs[i];
        for (int i = lane; i < F * 3 * nf; i += 32)
          {
            int64_t Fi = 0;
#pragma unroll
            for (int f = 0; f < F; ++f)
              if (f == i / (3 * nf))
                Fi = face_id[f];
            lam[i] = P.trace_state[Fi * 3 * nf + (i % (3 * nf))];
          }
        if (lane < F * 3)
          {
            const int f = lane / 3, b = lane % 3;
            int64_t   Fi = 0;
#pragma unroll
            for (int g = 0; g < F; ++g)
              if (g == f)
                Fi = face_id[g];
            taus[lane] = P.tau_table ? P.tau_table[(cell * F + f) * 3 + b] : P.tau[b];
            bcs[lane]  = (double)P.face_bc[Fi * 3 + b];
          }
        __syncwarp();

        // ------------------------------------ fields at quadrature points
        for (int i = lane; i < 3 * (DIM + 1) * nqc; i += 32)
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
        for (int i = lane; i < 3 * Fq; i += 32)
          {
            const int     b  = i / Fq;
            const int     fq = i % Fq;
            const int     f  = fq / nqf, qf = fq % nqf;
            const double  sg = (f & 1) ? 1. : -1.;
            const double *ph = phi_f + fq * nb;
            const double *cS = coef + (b * (DIM + 1) + DIM) * nb;
            const double *cW = coef + (b * (DIM + 1) + f / 2) * nb;
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
        __syncwarp();

        // --------------------- point coefficients and the flux residual
        for (int q = lane; q < nqc; q += 32)
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
        for (int i = lane; i < ncomp * DIM * nqc; i += 32)
          {
            const int     ce = i / (DIM * nqc);
            const int     b  = cmp_of(ce);
            const int     s  = (i / nqc) % DIM;
            const int     q  = i % nqc;
            const double *cS = coef + (b * (DIM + 1) + DIM) * nb;
            double        v  = -W0[(b * DIM + s) * nqc + q];
#pragma unroll
            for (int e = 0; e < nb; ++e)
              v += PW_c[(e * nqc + q) * DIM + s] * cS[e];
#pragma unroll
            for (int t = 0; t < Ft; ++t)
              v -= QW_c[(t * nqc + q) * DIM + s] * lam[((t / nf) * 3 + b) * nf + (t % nf)];
            Wrc[(ce * DIM + s) * nqc + q] = v;
          }
        for (int i = lane; i < ncomp * Fq; i += 32)
          {
            const int     ce = i / Fq;
            const int     b  = cmp_of(ce);
            const int     fq = i % Fq;
            const int     f = fq / nqf, qf = fq % nqf;
            const double *cS = coef + (b * (DIM + 1) + DIM) * nb;
            double        v  = -W0n[b * Fq + fq];
#pragma unroll
            for (int e = 0; e < nb; ++e)
              v += PW_f[(e * F + f) * nqf + qf] * cS[e];
#pragma unroll
            for (int t = 0; t < Ft; ++t)
              v -= QW_f[(t * F + f) * nqf + qf] * lam[((t / nf) * 3 + b) * nf + (t % nf)];
            Wrf[ce * Fq + fq] = v;
          }
        __syncwarp();

        // ------------------------------- channel coefficients per pair
        for (int i = lane; i < 9 * nqc; i += 32)
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
        for (int i = lane; i < 9 * Fq; i += 32)
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
        for (int i = lane; i < 3 * Fq; i += 32)
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
            if (bcs[f * 3 + b] == 2. && !thermo)
              {
                int64_t Fi = 0;
#pragma unroll
                for (int g = 0; g < F; ++g)
                  if (g == f)
                    Fi = face_id[g];
                rr += P.face_bc_val[(Fi * 3 + b) * nqf + qf];
              }
            ctc[i]  = c_;
            ctd[i]  = d_;
            tcS[i]  = s_;
            ttc[i]  = t_;
            rhsf[i] = rr;
          }
        __syncwarp();

        // ------------------------------------------ residual coefficients
        for (int i = lane; i < ncomp * nqc; i += 32)
          {
            const int    ce = i / nqc, q = i % nqc, b = cmp_of(ce);
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
                const double k_ = ka[(b * 3 + cmp_of(cp)) * nqc + q];
#pragma unroll
                for (int s = 0; s < DIM; ++s)
                  v1[s] -= k_ * Wrc[(cp * DIM + s) * nqc + q];
              }
            r0[ce * nqc + q] = v0;
#pragma unroll
            for (int s = 0; s < DIM; ++s)
              r1[(ce * nqc + q) * DIM + s] = v1[s];
          }
        for (int i = lane; i < ncomp * Fq; i += 32)
          {
            const int    ce = i / Fq, fq = i % Fq, b = cmp_of(ce);
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
              v -= rh[(b * 3 + cmp_of(cp)) * Fq + fq] * Wrf[cp * Fq + fq];
            rf[ce * Fq + fq] = v;
          }
        for (int t = lane; t < Nt; t += 32)
          {
            const int f = t / (ncomp * nf), ce = (t / nf) % ncomp, m = t % nf;
            const int b = cmp_of(ce);
            double    g = 0., fl = 0.;
            if (bcs[f * 3 + b] == 1.)
              {
                fl = 1.;
                if (!thermo)
                  {
                    int64_t Fi = 0;
#pragma unroll
                    for (int gg = 0; gg < F; ++gg)
                      if (gg == f)
                        Fi = face_id[gg];
#pragma unroll
                    for (int qf = 0; qf < nqf; ++qf)
                      g += fminvw[m * nqf + qf] *
                           (P.face_bc_val[(Fi * 3 + b) * nqf + qf] - tr0[(b * F + f) * nqf + qf]);
                  }
              }
            gv[t]  = g;
            dfl[t] = fl;
          }
        __syncwarp();

        // ---------------- right-hand sides R, one row per lane -> smem
        const bool act = lane < Ns;
        const int  ci  = act ? lane / nb : 0;
        const int  a   = act ? lane % nb : 0;
        const int  bi  = cmp_of(ci);
        if (act)
          {
            // residual column
            {
              const double *r0p = r0 + ci * nqc;
              const double *r1p = r1 + ci * nqc * DIM;
              const double *rfp = rf + ci * Fq;
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
              R[lane * ldr] = (JT)v;
            }
            // trace columns, one trial component at a time
            for (int cj = 0; cj < ncomp; ++cj)
              {
                const int     pr  = bi * 3 + cmp_of(cj);
                const JT     *kap = ka + pr * nqc;
                const JT     *rhp = rh + pr * Fq;
                double        acc[Ft];
#pragma unroll
                for (int t = 0; t < Ft; ++t)
                  acc[t] = 0.;
#pragma unroll
                for (int q = 0; q < nqc; ++q)
                  {
                    const double kq = (double)kap[q];
#pragma unroll
                    for (int s = 0; s < DIM; ++s)
                      {
                        const double w = kq * TLg[(q * DIM + s) * nb + a] * P.ih[s];
#pragma unroll
                        for (int t = 0; t < Ft; ++t)
                          acc[t] -= w * C.RQk[(q * DIM + s) * Ft + t];
                      }
                  }
#pragma unroll
                for (int fq = 0; fq < Fq; ++fq)
                  {
                    const double w = (double)rhp[fq] * TLf[fq * nb + a] * P.ih[fq / (nqf * 2)];
#pragma unroll
                    for (int t = 0; t < Ft; ++t)
                      acc[t] -= w * C.RQr[fq * Ft + t];
                  }
                if (cj == ci)
                  {
#pragma unroll
                    for (int f = 0; f < F; ++f)
#pragma unroll
                      for (int qf = 0; qf < nqf; ++qf)
                        {
                          const int    fq = f * nqf + qf;
                          const double w  = (double)ctc[bi * Fq + fq] * TLf[fq * nb + a];
#pragma unroll
                          for (int m = 0; m < nf; ++m)
                            acc[f * nf + m] += w * C.xi[qf * nf + m];
                        }
                  }
#pragma unroll
                for (int f = 0; f < F; ++f)
#pragma unroll
                  for (int m = 0; m < nf; ++m)
                    R[lane * ldr + 1 + (f * ncomp + cj) * nf + m] = (JT)acc[f * nf + m];
                if (two)
                  {
                    // drift columns are only used added to the trace columns:
                    // keep them combined (ct_cell + ct_drift)
#pragma unroll
                    for (int f = 0; f < F; ++f)
#pragma unroll
                      for (int m = 0; m < nf; ++m)
                        {
                          double d = acc[f * nf + m];
                          if (cj == ci)
#pragma unroll
                            for (int qf = 0; qf < nqf; ++qf)
                              {
                                const int fq = f * nqf + qf;
                                d += (double)ctd[bi * Fq + fq] * TLf[fq * nb + a] * C.xi[qf * nf + m];
                              }
                          R[lane * ldr + 1 + Nt + (f * ncomp + cj) * nf + m] = (JT)d;
                        }
                  }
              }
          }

        // ------------ S row per lane, in-place Gauss-Jordan inverse
        // lanes Ns..NSMAX-1 carry unit rows, so that the elimination always
        // runs over NSMAX columns (S padded to diag(S, I))
        JT srow[NSMAX];
#pragma unroll
        for (int j = 0; j < NSMAX; ++j)
          srow[j] = (lane >= Ns && lane == j) ? JT(1) : JT(0);
        if (act)
          {
#pragma unroll 1
            for (int cj = 0; cj < ncomp; ++cj)
              {
                const int     pr  = bi * 3 + cmp_of(cj);
                const JT     *alp = al + pr * nqc;
                const JT     *kap = ka + pr * nqc;
                const JT     *bep = be + pr * nqc * DIM;
                const JT     *gap = ga + pr * Fq;
                const JT     *rhp = rh + pr * Fq;
                double        acc[nb];
#pragma unroll
                for (int e = 0; e < nb; ++e)
                  acc[e] = 0.;
#pragma unroll
                for (int q = 0; q < nqc; ++q)
                  {
                    double lt = (double)alp[q] * TLc[q * nb + a];
                    double kt[DIM];
#pragma unroll
                    for (int s = 0; s < DIM; ++s)
                      {
                        const double tg = TLg[(q * DIM + s) * nb + a];
                        lt += (double)bep[q * DIM + s] * tg;
                        kt[s] = (double)kap[q] * tg * P.ih[s];
                      }
#pragma unroll
                    for (int e = 0; e < nb; ++e)
                      {
                        acc[e] += lt * C.phi_c[q * nb + e];
#pragma unroll
                        for (int s = 0; s < DIM; ++s)
                          acc[e] += kt[s] * C.RTk[(q * DIM + s) * nb + e];
                      }
                  }
#pragma unroll
                for (int fq = 0; fq < Fq; ++fq)
                  {
                    const double tf = TLf[fq * nb + a];
                    const double g_ = (double)gap[fq] * tf, r_ = (double)rhp[fq] * tf * P.ih[fq / (nqf * 2)];
#pragma unroll
                    for (int e = 0; e < nb; ++e)
                      acc[e] += g_ * C.phi_f[fq * nb + e] + r_ * C.RTr[fq * nb + e];
                  }
                // block cj of the row (selects: no dynamic register index)
#pragma unroll
                for (int k = 0; k < NSMAX; ++k)
                  if (k / nb == cj)
                    srow[k] = (JT)acc[k % nb];
              }
          }
        // ---------------------------------------- Gauss-Jordan inverse
        // Row equilibration: S' = D S with D = diag(1/max|row|).  The sweep
        // below inverts S'; S^-1 = S'^-1 D, so column k of the inverse is
        // scaled by the factor of row p_k before it multiplies R.
        JT rscale;
        {
          JT mx = 0;
#pragma unroll
          for (int j = 0; j < NSMAX; ++j)
            mx = fmax(mx, fabs(srow[j]));
          rscale = (mx > JT(0)) ? JT(1) / mx : JT(1);
#pragma unroll
          for (int j = 0; j < NSMAX; ++j)
            srow[j] *= rscale;
        }
        // Sweep (exchange) form of Gauss-Jordan with virtual partial
        // pivoting: step j exchanges unknown j with equation p_j.  The row is
        // rotated left by one register per step, so column j sits in srow[0]
        // at step j and NSMAX steps bring every column back to its place.
        // Afterwards lane p_j holds row j of S'^-1, whose column k belongs to
        // equation p_k.
        // Pivot choice: one warp max-reduction of a 32-bit key made of the
        // high word of |S'_ij| (sign, exponent and 20 mantissa bits) with the
        // low 5 bits replaced by 31 - lane: the pivot is within 2^-15 of the
        // largest candidate, ties go to the lowest lane.  The pivot row is
        // broadcast by shuffles, element by element as the update uses it.
        static_assert(NSMAX < 32, "key 0 marks used lanes");
        bool    used  = lane >= NSMAX;
        int     mypos = 0;
        bool    sing  = false;
#pragma unroll 1
        for (int j = 0; j < NSMAX; ++j)
          {
            unsigned key = 0u;
            if (!used)
              {
                const unsigned hi = pivot_key_bits(srow[0]);
                key = (hi & ~31u) | (31u - (unsigned)lane);
              }
            const unsigned kmax = __reduce_max_sync(0xffffffffu, key);
            const int      bl   = 31 - (int)(kmax & 31u);
            const bool     me   = lane == bl;
            const JT pj = __shfl_sync(0xffffffffu, srow[0], bl);
            sing |= kmax < 32u || !isfinite(pj);
            const JT hr = (pj != JT(0)) ? JT(1) / pj : JT(0);
            const JT l  = srow[0] * hr;
#pragma unroll
            for (int k = 1; k < NSMAX; ++k)
              {
                const JT pk = __shfl_sync(0xffffffffu, srow[k], bl);
                srow[k - 1]     = me ? -pk * hr : srow[k] - l * pk;
              }
            srow[NSMAX - 1] = me ? hr : l;
            if (me)
              {
                used  = true;
                mypos = j;
              }
            if (lane == 0)
              piv[j] = bl;
            __syncwarp();
          }
        if (sing && lane == 0)
          atomicExch(P.status, 3);
        __syncwarp();
        // fold the row scaling of equation p_k into column k
        {
          JT dsc[NSMAX];
#pragma unroll
          for (int k = 0; k < NSMAX; ++k)
            dsc[k] = __shfl_sync(0xffffffffu, rscale, piv[k]);
#pragma unroll
          for (int k = 0; k < NSMAX; ++k)
            srow[k] *= dsc[k];
        }

        // ---------- Y = S^-1 R on the FP64 tensor path, written back over R
        {
          constexpr int MP = (NSMAX + 7) / 8 * 8;
          constexpr int KP = (NSMAX + 3) / 4 * 4;
          constexpr int KS = sinv_stride_for(NSMAX, (int)sizeof(JT));
          JT           *Sv = reinterpret_cast<JT *>(coef); // the coefficient block is dead here
          for (int idx = lane; idx < MP * KS; idx += 32)
            Sv[idx] = 0.;
          __syncwarp();
          if (act)
            {
#pragma unroll
              for (int k = 0; k < NSMAX; ++k)
                Sv[mypos * KS + k] = srow[k];
            }
          __syncwarp();
          const int g = lane >> 2, tq = lane & 3;
          for (int n0 = 0; n0 < ncol; n0 += 8)
            {
              const int col = n0 + g;
              double    bf[KP / 4];
#pragma unroll
              for (int ks = 0; ks < KP / 4; ++ks)
                {
                  const int kk = ks * 4 + tq;
                  bf[ks] = (kk < Ns && col < ncol) ? (double)R[piv[kk] * ldr + col] : 0.;
                }
              double acc[MP / 8][2];
#pragma unroll
              for (int mt = 0; mt < MP / 8; ++mt)
                {
                  acc[mt][0] = acc[mt][1] = 0.;
#pragma unroll
                  for (int ks = 0; ks < KP / 4; ++ks)
                    dmma8x8x4(acc[mt][0], acc[mt][1], (double)Sv[(mt * 8 + g) * KS + ks * 4 + tq],
                              bf[ks]);
                }
              __syncwarp(); // every lane has read this block of R columns
#pragma unroll
              for (int mt = 0; mt < MP / 8; ++mt)
                {
                  const int row = mt * 8 + g;
#pragma unroll
                  for (int e = 0; e < 2; ++e)
                    {
                      const int c = n0 + 2 * tq + e;
                      if (row < Ns && c < ncol)
                        R[row * ldr + c] = (JT)acc[mt][e];
                    }
                }
              __syncwarp();
            }
        }
        JT *const Y = R;

        // ------------------------ keep Y for the reconstruction [col][row]
        {
          double   *yc  = P.ycache + cell * (int64_t)Ns * P.ycols;
          const int tot = Ns * P.ycols;
          int       row = lane % Ns, col = lane / Ns;
          for (int idx = lane; idx < tot; idx += 32)
            {
              yc[idx] = Y[row * ldr + col];
              row += 32;
              while (row >= Ns)
                {
                  row -= Ns;
                  ++col;
                }
            }
        }
        // combined residual column with the Dirichlet columns folded in
        for (int j = lane; j < Ns; j += 32)
          {
            double acc = Y[j * ldr];
            for (int t = 0; t < Nt; ++t)
              if (dfl[t] != 0.)
                acc -= gv[t] * Y[j * ldr + colC + t];
            Yc[j] = acc;
          }
        __syncwarp(); // the coefficient arrays are dead from here on

        // ------------- trace-row data: face weights, H = Wrf - Dirichlet flux
        for (int idx = lane; idx < ncomp * Fq; idx += 32)
          {
            const int cp = idx / Fq, fq = idx % Fq;
            double    h  = Wrf[idx];
#pragma unroll
            for (int ft = 0; ft < F; ++ft)
#pragma unroll
              for (int mt = 0; mt < nf; ++mt)
                {
                  const int t = (ft * ncomp + cp) * nf + mt;
                  if (dfl[t] != 0.)
                    h -= gv[t] * RQr[fq * Ft + ft * nf + mt];
                }
            Hs[idx] = h;
          }
        __syncwarp();
        for (int i = lane; i < Nt; i += 32)
          {
            const int fi = i / (ncomp * nf), ci2 = (i / nf) % ncomp, mi = i % nf;
            const int b  = cmp_of(ci2);
            double    z  = 0.;
#pragma unroll
            for (int qf = 0; qf < nqf; ++qf)
              {
                const int    fq = fi * nqf + qf;
                const double w  = w_f[fq] * xi[qf * nf + mi];
                if (!RW)
                  {
                    rS[i * nqf + qf] = w * tcS[b * Fq + fq];
                    rD[i * nqf + qf] = w * ttc[b * Fq + fq];
                  }
                z += w * rhsf[b * Fq + fq];
                for (int cp = 0; cp < ncomp; ++cp)
                  {
                    const double tw = w * tcW[(b * 3 + cmp_of(cp)) * Fq + fq];
                    if (!RW)
                      rA[(i * 3 + cp) * nqf + qf] = tw;
                    z += tw * Hs[cp * Fq + fq];
                  }
              }
            rZ[i] = z;
          }
        __syncwarp();

        // --------- reduced trace operator T = tc_c + tc_W P, stored [j][i]
        for (int idx = lane; idx < Nt * ncomp; idx += 32)
          {
            const int i = idx / ncomp, cj = idx - i * ncomp;
            const int fi = i / (ncomp * nf), ci2 = (i / nf) % ncomp;
            double    wa[nqf], ws_[nqf];
#pragma unroll
            for (int qf = 0; qf < nqf; ++qf)
              {
                if (RW)
                  {
                    const int    fq = fi * nqf + qf, bb = cmp_of(ci2);
                    const double w  = w_f[fq] * xi[qf * nf + i % nf];
                    wa[qf]          = w * tcW[(bb * 3 + cmp_of(cj)) * Fq + fq];
                    ws_[qf]         = (cj == ci2) ? w * tcS[bb * Fq + fq] : 0.;
                  }
                else
                  {
                    wa[qf]  = rA[(i * 3 + cj) * nqf + qf];
                    ws_[qf] = (cj == ci2) ? rS[i * nqf + qf] : 0.;
                  }
              }
#pragma unroll
            for (int e = 0; e < nb; ++e)
              {
                double v = 0.;
#pragma unroll
                for (int qf = 0; qf < nqf; ++qf)
                  {
                    const int fq = fi * nqf + qf;
                    v += wa[qf] * RTr[fq * nb + e] + ws_[qf] * phi_f[fq * nb + e];
                  }
                Trs[(cj * nb + e) * Nt + i] = v;
              }
          }
        __syncwarp();

        // ------------------------------------- right-hand side and flags
        for (int i = lane; i < Nt; i += 32)
          {
            const bool rowD = dfl[i] != 0.;
            double     r    = 0.;
            if (!rowD)
              {
                for (int j = 0; j < Ns; ++j)
                  r += Trs[j * Nt + i] * Yc[j];
                r += rZ[i];
              }
            P.rhs[cell * Nt + i]   = r;
            P.dflag[cell * Nt + i] = rowD ? 1 : 0;
            P.dval[cell * Nt + i]  = gv[i];
          }

        // ---- tt = T Y_comb + tc_W Q_t + face block, FP64 tensor-path tiles
        {
          constexpr int NTM    = F * 3 * nf;
          constexpr int NNT    = (NTM + 7) / 8; // column tiles (all enabled components)
          constexpr int KP     = (NSMAX + 3) / 4 * 4;
          const int     g      = lane >> 2, tq = lane & 3;
          double       *tt_out = P.tt + cell * (int64_t)Nt * Nt;
          // this lane's output columns t = 8 nt + 2 tq + e, decoded once:
          // face | component << 4 | node << 8 | (usable column) << 15
          int cm[NNT][2];
#pragma unroll
          for (int nt = 0; nt < NNT; ++nt)
#pragma unroll
            for (int e = 0; e < 2; ++e)
              {
                const int t  = nt * 8 + 2 * tq + e;
                const int tt = t < Nt ? t : 0;
                cm[nt][e]    = (tt / (ncomp * nf)) | (((tt / nf) % ncomp) << 4) | ((tt % nf) << 8) |
                            ((t < Nt && dfl[tt] == 0.) ? (1 << 15) : 0);
              }
          for (int m0 = 0; m0 < Nt; m0 += 8)
            {
              const int i = m0 + g; // output row of this lane
              double    d[NNT][2];
#pragma unroll
              for (int nt = 0; nt < NNT; ++nt)
                d[nt][0] = d[nt][1] = 0.;
#pragma unroll
              for (int ks = 0; ks < KP / 4; ++ks)
                {
                  const int    j  = ks * 4 + tq;
                  const double av = (i < Nt && j < Ns) ? Trs[j * Nt + i] : 0.;
#pragma unroll
                  for (int nt = 0; nt < NNT; ++nt)
                    {
                      const int    tb = nt * 8 + g; // B-fragment column
                      const double bv = (j < Ns && tb < Nt) ? Y[j * ldr + colC + tb] : 0.;
                      dmma8x8x4(d[nt][0], d[nt][1], av, bv);
                    }
                }
              if (i >= Nt)
                continue;
              const int  fi  = i / (ncomp * nf), ci2 = (i / nf) % ncomp;
              const bool rok = dfl[i] == 0.;
              const JT    *rAi = rA + i * 3 * nqf, *rDi = rD + i * nqf;
              // 3D FP64: the row's face weights, times the coefficients below
              double wi[nqf];
              int    bi3 = 0;
              if (RW)
                {
                  bi3 = cmp_of(ci2);
#pragma unroll
                  for (int qf = 0; qf < nqf; ++qf)
                    wi[qf] = w_f[fi * nqf + qf] * xi[qf * nf + i % nf];
                }
#pragma unroll
              for (int nt = 0; nt < NNT; ++nt)
#pragma unroll
                for (int e = 0; e < 2; ++e)
                  {
                    const int t = nt * 8 + 2 * tq + e;
                    if (t >= Nt)
                      continue;
                    const int c  = cm[nt][e];
                    double    o  = 0.;
                    if (rok && (c >> 15))
                      {
                        const int ft = c & 15, ct = (c >> 4) & 15, mt = (c >> 8) & 127;
                        const int tqq = ft * nf + mt;
                        double    z   = d[nt][e];
#pragma unroll
                        for (int qf = 0; qf < nqf; ++qf)
                          {
                            const double ra =
                              RW ? wi[qf] * tcW[(bi3 * 3 + cmp_of(ct)) * Fq + fi * nqf + qf]
                                 : (double)rAi[ct * nqf + qf];
                            z += ra * RQr[(fi * nqf + qf) * Ft + tqq];
                          }
                        if (ft == fi && ct == ci2)
#pragma unroll
                          for (int qf = 0; qf < nqf; ++qf)
                            {
                              const double rd =
                                RW ? wi[qf] * ttc[bi3 * Fq + fi * nqf + qf] : (double)rDi[qf];
                              z += rd * xi[qf * nf + mt];
                            }
                        o = z;
                      }
                    tt_out[(int64_t)i * Nt + t] = o;
                  }
            }
        }
        __syncwarp();
      }
  }

  template <int DIM, int K, typename JT = double>
  __global__ void __launch_bounds__(Condense3MaxWPB * 32, sizeof(JT) == 8 ? 1 : 2)
  condense3_kernel(const KParams P, const __grid_constant__ CTab<DIM, K> C)
  {
    extern __shared__ __align__(16) double smem[];
    __shared__ int    piv3[Condense3MaxWPB][3 * Dims<DIM, K>::nb];
    __shared__ double rqr_s[CTab<DIM, K>::Fq * CTab<DIM, K>::Ft];
    for (int i = threadIdx.x; i < CTab<DIM, K>::Fq * CTab<DIM, K>::Ft; i += blockDim.x)
      rqr_s[i] = P.tables[P.to.RQr + i];
    __syncthreads();
    const int      warp = threadIdx.x >> 5;
    const int      wpb  = blockDim.x >> 5;
    const Ws3Off   wo   = ws3_layout(DIM, Dims<DIM, K>::nb, Dims<DIM, K>::nf, P.ncomp, P.ncol, (int)sizeof(JT));
    condense3_cells<DIM, K, JT>(P, C, smem + warp * wo.total, piv3[warp],
                                P.cell0 + (int64_t)blockIdx.x * wpb + warp, P.ncells,
                                (int64_t)gridDim.x * wpb, rqr_s);
  }
} // namespace ddhdg
