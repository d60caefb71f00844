// Dense kernels of the nested-dissection trace solve on the FP64 tensor path
// (mma.sync m8n8k4 f64), for the fronts of one batch at once:
//
//   nd_trinv_kernel   inverses of the 32 x 32 diagonal blocks of the LU
//                     factors L (unit lower) and U (upper) of F_EE
//   nd_trsm_kernel    W = U^-1 L^-1 [F_EK | r_E] in place, by 32-row blocks:
//                     W_i = Linv_ii (B_i - sum_j<i L_ij W_j), then
//                     X_i = Uinv_ii (W_i - sum_j>i U_ij X_j)
//   nd_gemm_kernel    the Schur update F_KK -= F_KE W (64 x 64 tiles)
//
// They replace the library triangular solves and products of the fronts
// that are factorised by an LU with partial pivoting (own or cuSOLVER),
// all fronts of a batch in one launch each.  Fronts are column-major with
// leading dimension nF; the per-front blocks come from the batch's pointer
// table (F_EE, [F_EK | r_E], F_KE, F_KK).  Ragged edges are zero-padded in
// shared memory (identity on the padded diagonal of the inverted blocks).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "hdg_condense3.cuh" // dmma8x8x4

namespace ddhdg
{
  constexpr int NDTB = 32; // diagonal block of the triangular solves

  // ------------------------------------------------- diagonal-block inverses
  // grid (blocks per front, fronts), 64 threads: warp 0 inverts the unit
  // lower block of L, warp 1 the upper block of U.  tinv[(f * nblk + blk) *
  // 2 + which][32 x 32] column-major.
  __global__ void __launch_bounds__(64)
  nd_trinv_kernel(int nE, int ld, double *const *pEE, double *tinv)
  {
    __shared__ double S[2][NDTB][NDTB + 1];
    const int    nblk = (nE + NDTB - 1) / NDTB;
    const int    blk = blockIdx.x, f = blockIdx.y;
    const int    w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int    r0 = blk * NDTB;
    const double *F = pEE[f];
    // the diagonal block, identity beyond nE
    for (int idx = lane; idx < NDTB * NDTB; idx += 32)
      {
        const int r = idx % NDTB, c = idx / NDTB;
        double    v;
        if (r0 + r < nE && r0 + c < nE)
          v = F[(int64_t)(r0 + c) * ld + r0 + r];
        else
          v = (r == c) ? 1. : 0.;
        S[w][r][c] = v;
      }
    __syncwarp();
    const int c = lane; // this lane's column of the inverse
    double    x[NDTB];
    if (w == 0)
      {
        // unit lower: x_r = -sum_{c <= s < r} L_rs x_s
#pragma unroll
        for (int r = 0; r < NDTB; ++r)
          {
            double v = (r == c) ? 1. : 0.;
            if (r > c)
#pragma unroll
              for (int s = 0; s < r; ++s)
                if (s >= c)
                  v -= S[0][r][s] * x[s];
            x[r] = v;
          }
      }
    else
      {
        // upper: x_r = -(sum_{r < s <= c} U_rs x_s) / U_rr, x_c = 1 / U_cc
#pragma unroll
        for (int r = NDTB - 1; r >= 0; --r)
          {
            double v = 0.;
            if (r == c)
              v = 1. / S[1][r][r];
            else if (r < c)
              {
#pragma unroll
                for (int s = r + 1; s < NDTB; ++s)
                  if (s <= c)
                    v -= S[1][r][s] * x[s];
                v /= S[1][r][r];
              }
            x[r] = v;
          }
      }
    double *out = tinv + ((int64_t)(f * nblk + blk) * 2 + w) * NDTB * NDTB;
#pragma unroll
    for (int r = 0; r < NDTB; ++r)
      out[c * NDTB + r] = x[r];
  }

  // ------------------------------------------------------ triangular solves
  // acc (warp's 8 x 32 strip of a 32 x 32 block) -= / = Ts (32 x 32) x Ws
  // (32 x 32); lane layout of mma.m8n8k4: A[l/4][l%4], B[l%4][l/4],
  // D[l/4][2 (l%4) + e]
  __device__ __forceinline__ void
  nd_blk_mma(double (&acc)[4][2], const double (*Ts)[NDTB + 4], const double (*Ws)[NDTB + 8], int warp,
             int lane)
  {
#pragma unroll
    for (int kk = 0; kk < NDTB / 4; ++kk)
      {
        const double a = Ts[warp * 8 + (lane >> 2)][kk * 4 + (lane & 3)];
#pragma unroll
        for (int j = 0; j < 4; ++j)
          dmma8x8x4(acc[j][0], acc[j][1], a, Ws[kk * 4 + (lane & 3)][j * 8 + (lane >> 2)]);
      }
  }

  // grid (column tiles of 32, fronts), 128 threads.  B = [F_EK | r_E] rows
  // 0..nE-1 of front f (pB[f]), ncols columns; overwritten by W.
  __global__ void __launch_bounds__(128)
  nd_trsm_kernel(int nE, int ncols, int ld, double *const *pEE, double *const *pB, const double *tinv)
  {
    __shared__ __align__(16) double Ts[NDTB][NDTB + 4];
    __shared__ __align__(16) double Ws[NDTB][NDTB + 8];
    const int     nblk = (nE + NDTB - 1) / NDTB;
    const int     f    = blockIdx.y;
    const int     c0   = blockIdx.x * NDTB;
    const int     nc   = min(NDTB, ncols - c0);
    const int     tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const double *LU = pEE[f];
    double       *B  = pB[f] + (int64_t)c0 * ld;
    const double *TI = tinv + (int64_t)f * nblk * 2 * NDTB * NDTB;

    auto load_T = [&](int r0, int k0) { // block of the factor at (r0, k0)
      for (int idx = tid; idx < NDTB * NDTB; idx += 128)
        {
          const int r = idx % NDTB, k = idx / NDTB;
          Ts[r][k]    = (r0 + r < nE && k0 + k < nE) ? LU[(int64_t)(k0 + k) * ld + r0 + r] : 0.;
        }
    };
    auto load_inv = [&](int blk, int which) {
      const double *src = TI + ((int64_t)blk * 2 + which) * NDTB * NDTB;
      for (int idx = tid; idx < NDTB * NDTB; idx += 128)
        Ts[idx % NDTB][idx / NDTB] = src[idx];
    };
    auto load_W = [&](int r0) { // rows r0.. of this column tile
      for (int idx = tid; idx < NDTB * NDTB; idx += 128)
        {
          const int k = idx % NDTB, c = idx / NDTB;
          Ws[k][c]    = (r0 + k < nE && c < nc) ? B[(int64_t)c * ld + r0 + k] : 0.;
        }
    };
    auto acc_load = [&](double (&acc)[4][2], int r0) {
      const int r = r0 + warp * 8 + (lane >> 2);
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int e = 0; e < 2; ++e)
          {
            const int c  = j * 8 + 2 * (lane & 3) + e;
            acc[j][e]    = (r < nE && c < nc) ? B[(int64_t)c * ld + r] : 0.;
          }
    };
    auto acc_to_W = [&](const double (&acc)[4][2]) {
      const int r = warp * 8 + (lane >> 2);
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int e = 0; e < 2; ++e)
          Ws[r][j * 8 + 2 * (lane & 3) + e] = acc[j][e];
    };
    auto acc_store = [&](const double (&acc)[4][2], int r0) {
      const int r = r0 + warp * 8 + (lane >> 2);
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int e = 0; e < 2; ++e)
          {
            const int c = j * 8 + 2 * (lane & 3) + e;
            if (r < nE && c < nc)
              B[(int64_t)c * ld + r] = acc[j][e];
          }
    };

    // forward: W_i = Linv_ii (B_i - sum_{j<i} L_ij W_j)
    for (int i = 0; i < nblk; ++i)
      {
        double acc[4][2];
        acc_load(acc, i * NDTB);
        for (int j = 0; j < i; ++j)
          {
            __syncthreads();
            load_T(i * NDTB, j * NDTB);
            load_W(j * NDTB);
            __syncthreads();
            double p[4][2] = {};
            nd_blk_mma(p, Ts, Ws, warp, lane);
#pragma unroll
            for (int a = 0; a < 4; ++a)
              {
                acc[a][0] -= p[a][0];
                acc[a][1] -= p[a][1];
              }
          }
        __syncthreads();
        acc_to_W(acc);
        load_inv(i, 0);
        __syncthreads();
        double o[4][2] = {};
        nd_blk_mma(o, Ts, Ws, warp, lane);
        acc_store(o, i * NDTB);
        __threadfence_block();
      }
    // backward: X_i = Uinv_ii (W_i - sum_{j>i} U_ij X_j)
    for (int i = nblk - 1; i >= 0; --i)
      {
        __syncthreads();
        double acc[4][2];
        acc_load(acc, i * NDTB);
        for (int j = i + 1; j < nblk; ++j)
          {
            __syncthreads();
            load_T(i * NDTB, j * NDTB);
            load_W(j * NDTB);
            __syncthreads();
            double p[4][2] = {};
            nd_blk_mma(p, Ts, Ws, warp, lane);
#pragma unroll
            for (int a = 0; a < 4; ++a)
              {
                acc[a][0] -= p[a][0];
                acc[a][1] -= p[a][1];
              }
          }
        __syncthreads();
        acc_to_W(acc);
        load_inv(i, 1);
        __syncthreads();
        double o[4][2] = {};
        nd_blk_mma(o, Ts, Ws, warp, lane);
        acc_store(o, i * NDTB);
        __threadfence_block();
      }
  }

  // --------------------------------------------------------------- C -= A B
  constexpr int NDGM = 64, NDGN = 64, NDGK = 16;
  constexpr int NDGLA = NDGM + 8;  // As[k][m] row stride (doubles)
  constexpr int NDGLB = NDGK + 4;  // Bs[n][k] row stride

  __device__ __forceinline__ void
  nd_cp_async8(double *dst, const double *src, bool valid)
  {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    const int      n = valid ? 8 : 0; // 0 source bytes: the 8 bytes are zero-filled
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(d), "l"(src), "r"(n));
  }

  // grid (tiles of C, fronts), 128 threads (2 x 2 warps of 32 x 32).
  // C (m x n) -= A (m x k) B (k x n), column-major, leading dimension ld.
  __global__ void __launch_bounds__(128)
  nd_gemm_kernel(int m, int n, int k, int ld, double *const *Ap, double *const *Bp, double *const *Cp)
  {
    __shared__ __align__(16) double As[2][NDGK][NDGLA];
    __shared__ __align__(16) double Bs[2][NDGN][NDGLB];
    const int     tiles_m = (m + NDGM - 1) / NDGM;
    const int     m0 = (blockIdx.x % tiles_m) * NDGM, n0 = (blockIdx.x / tiles_m) * NDGN;
    const int     f  = blockIdx.y;
    const double *A  = Ap[f];
    const double *Bm = Bp[f];
    double       *C  = Cp[f];
    const int     tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int     wm = (warp & 1) * 32, wn = (warp >> 1) * 32;
    const int     nchunk = (k + NDGK - 1) / NDGK;

    auto issue = [&](int chunk, int buf) {
      const int k0 = chunk * NDGK;
#pragma unroll
      for (int q = 0; q < NDGM * NDGK / 128; ++q)
        {
          const int  idx = tid + 128 * q;
          const int  mm = idx % NDGM, kk = idx / NDGM;
          const bool ok = m0 + mm < m && k0 + kk < k;
          nd_cp_async8(&As[buf][kk][mm], ok ? A + (int64_t)(k0 + kk) * ld + m0 + mm : A, ok);
        }
#pragma unroll
      for (int q = 0; q < NDGN * NDGK / 128; ++q)
        {
          const int  idx = tid + 128 * q;
          const int  kk = idx % NDGK, nn = idx / NDGK;
          const bool ok = n0 + nn < n && k0 + kk < k;
          nd_cp_async8(&Bs[buf][nn][kk], ok ? Bm + (int64_t)(n0 + nn) * ld + k0 + kk : Bm, ok);
        }
      asm volatile("cp.async.commit_group;" ::: "memory");
    };

    double acc[4][4][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j)
        acc[i][j][0] = acc[i][j][1] = 0.;
    issue(0, 0);
    for (int c = 0; c < nchunk; ++c)
      {
        const int buf = c & 1;
        if (c + 1 < nchunk)
          {
            issue(c + 1, buf ^ 1);
            asm volatile("cp.async.wait_group 1;" ::: "memory");
          }
        else
          asm volatile("cp.async.wait_group 0;" ::: "memory");
        __syncthreads();
#pragma unroll
        for (int ks = 0; ks < NDGK / 4; ++ks)
          {
            double a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i)
              a[i] = As[buf][ks * 4 + (lane & 3)][wm + i * 8 + (lane >> 2)];
#pragma unroll
            for (int j = 0; j < 4; ++j)
              b[j] = Bs[buf][wn + j * 8 + (lane >> 2)][ks * 4 + (lane & 3)];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
              for (int j = 0; j < 4; ++j)
                dmma8x8x4(acc[i][j][0], acc[i][j][1], a[i], b[j]);
          }
        __syncthreads();
      }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int e = 0; e < 2; ++e)
          {
            const int r = m0 + wm + i * 8 + (lane >> 2);
            const int col = n0 + wn + j * 8 + 2 * (lane & 3) + e;
            if (r < m && col < n)
              C[(int64_t)col * ld + r] -= acc[i][j][e];
          }
  }
} // namespace ddhdg
