// Shared definitions of the device kernels (sm_100a, FP64) and the cell
// reconstruction kernel.  The per-cell condensation kernel is in
// hdg_condense.cuh.
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
      Q, minv, TLc, TLg, TLf, RTk, RTr, RQk, RQr, total;
  };

  struct KParams
  {
    // mesh
    int     n[3];
    int64_t ncells; // cells [cell0, ncells) are processed by a launch
    int64_t cell0;
    int64_t face_off[3];
    int     face_ext[3][3];
    double  ih[3]; // 1 / cell size per axis (scales the unit-cell CTab operators)
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
    int stage; // 1: copy the tables to shared memory, 0: read them from L1/L2
    // state
    const double *cell_state, *trace_state;
    // outputs
    double  *tt, *rhs, *dval, *ycache;
    double  *rscratch; // per-CTA R blocks when they do not fit in shared memory, or null
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

  __device__ inline int64_t
  face_index(const KParams &P, int64_t cell, int f, int dim)
  {
    // 32-bit divisions: contexts hold fewer than 2^31 cells
    int            ci[3];
    const unsigned c  = (unsigned)cell;
    const unsigned n0 = (unsigned)P.n[0], n1 = (unsigned)P.n[1];
    const unsigned q  = c / n0;
    ci[0]             = (int)(c - q * n0);
    ci[1]             = (int)(q % n1);
    ci[2]             = (int)(q / n1);
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

  // --------------------------------------------------------- reconstruct
  // Cell update from the trace update: du = Y0 - Y_t dlam for the scalar
  // unknowns, and the flux unknowns from the (linear) flux rows,
  // W_new = P u_new - Q lam_new, i.e. dW = P(u0+du) - W0 - Q(lam0+dlam).
  //
  // The body: the whole CTA stages P and Q, then every warp works through the
  // cells cell_begin + warp * warp_step, then + cell_step, ... < cell_end.
  template <int DIM, int K>
  __device__ __forceinline__ void
  reconstruct_cells(const KParams &P, const double *__restrict__ dtrace,
                    double *__restrict__ dcell, double *smem, int64_t cell_begin,
                    int64_t warp_step, int64_t cell_end, int64_t cell_step)
  {
    using Dm          = Dims<DIM, K>;
    constexpr int nb  = Dm::nb;
    constexpr int nf  = Dm::nf;
    constexpr int F   = Dm::F;
    constexpr int NCA = Dm::Nc_all;
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
    const int     wsz = Ns + 2 * F * 3 * nf + nb + Nt;
    double *ws   = smem + ((nPQ + 1) & ~1) + warp * ((wsz + 1) & ~1);
    double *du   = ws;
    double *dl   = ws + Ns;          // [F][3][nf] trace update
    double *lnew = dl + F * 3 * nf;  // [F][3][nf] lam0 + dlam
    double *unew = lnew + F * 3 * nf;
    double *dlr  = unew + nb;        // [Nt] trace update, restricted order

    for (int64_t cell = cell_begin + warp * warp_step; cell < cell_end; cell += cell_step)
      {
        // the cell's face ids: one lane per face, then shuffled (the loop
        // runs the same number of times on every lane)
        const int64_t my_face = face_index(P, cell, lane < F ? lane : 0, DIM);
        for (int i0 = 0; i0 < F * 3 * nf; i0 += 32)
          {
            const int     i  = i0 + lane;
            const bool    in = i < F * 3 * nf;
            const int64_t Fi = __shfl_sync(0xffffffffu, my_face, in ? i / (3 * nf) : 0);
            if (in)
              {
                const double d = dtrace[Fi * 3 * nf + (i % (3 * nf))];
                dl[i]          = d;
                lnew[i]        = P.trace_state[Fi * 3 * nf + (i % (3 * nf))] + d;
              }
          }
        __syncwarp();
        for (int t = lane; t < Nt; t += 32)
          {
            const int f  = t / (ncomp * nf);
            const int ce = (t / nf) % ncomp;
            const int b  = ce == 0 ? P.comps[0] : (ce == 1 ? P.comps[1] : P.comps[2]);
            dlr[t]       = dl[(f * 3 + b) * nf + t % nf];
          }
        __syncwarp();
        const double *Y = P.ycache + cell * (int64_t)Ns * P.ycols;
        for (int i = lane; i < Ns; i += 32)
          {
            const double *Yi = Y + Ns + i;
            double        v0 = Y[i], v1 = 0., v2 = 0., v3 = 0.;
            int           t  = 0;
            for (; t + 4 <= Nt; t += 4)
              {
                v0 -= Yi[(t + 0) * Ns] * dlr[t + 0];
                v1 -= Yi[(t + 1) * Ns] * dlr[t + 1];
                v2 -= Yi[(t + 2) * Ns] * dlr[t + 2];
                v3 -= Yi[(t + 3) * Ns] * dlr[t + 3];
              }
            for (; t < Nt; ++t)
              v0 -= Yi[t * Ns] * dlr[t];
            du[i] = (v0 + v1) + (v2 + v3);
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

  template <int DIM, int K>
  __global__ void __launch_bounds__(256, 8) // 8 CTAs per SM: memory-latency bound
  reconstruct_kernel(const KParams P, const double *__restrict__ dtrace,
                     double *__restrict__ dcell)
  {
    extern __shared__ double smem[];
    reconstruct_cells<DIM, K>(P, dtrace, dcell, smem, P.cell0 + (int64_t)blockIdx.x * P.wpb, 1,
                              P.ncells, (int64_t)gridDim.x * P.wpb);
  }
} // namespace ddhdg
