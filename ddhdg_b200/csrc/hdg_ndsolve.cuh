// Global trace solve of the HDG system on a structured mesh (sm_100a, FP64).
//
// The global trace matrix is the sum over cells of the condensed per-cell
// blocks tt (copy_local_to_global, src/np_solver.cpp:1293-1322, with the
// Dirichlet rows replaced by identity rows).  The reference factorises it
// with UMFPACK (src/np_solver.cpp:1326-1354).  Here it is factorised
// directly from the per-cell blocks by nested dissection: the cell grid is
// bisected recursively (longest axis first) and every tree node is a dense
// front over the trace dofs of the faces on its split plane (eliminated
// there) and of the faces on its boundary (kept for the parent).
//
//   leaves    one front per cell: the cell's block tt, with the faces on the
//             physical boundary eliminated (Dirichlet dofs are identity rows)
//   upward    a node's front is the extend-add of its two children's Schur
//             complements; LU with partial pivoting of the eliminated block,
//             W = F_EE^-1 [F_EK | r_E], Schur update F_KK -= F_KE W
//   downward  x_E = y_E - W x_K from the root to the leaves
//
// Fronts of one height and one shape are processed as one batch:
//   <= 36 eliminated dofs   one fused kernel, a CTA per front (LU, W and the
//                           Schur update); above the leaves, while the front
//                           fits, it is also assembled in shared memory
//   37..72                  a CTA per front for the LU and W, the Schur update
//                           as one tensor-path GEMM launch for the batch
//   up to 383               own LU, a CTA per front (all fronts at once), then
//                           batched cuBLAS triangular solves and the GEMM launch
//   >= 384 (few fronts)     cuSOLVER LU and cuBLAS triangular solves per front
//                           on side streams, then the GEMM launch
// Above the smallest fronts, the Schur updates F_KK -= F_KE W and the
// triangular solves for W are cuBLAS calls by default.  Their tensor-path
// counterparts (hdg_ndblas.cuh: nd_gemm_kernel for all fronts of a batch in
// one launch, DDHDG_ND_OWN_GEMM=1; 32-row block substitution with inverted
// diagonal blocks, DDHDG_ND_OWN_TRSM=1) give the same solution to round-off
// and measured slower at 1.18M dofs.
// The numeric sequence is captured in a CUDA graph on the second call with
// the same buffers and replayed afterwards.  Before the factorisation the
// rows are equilibrated: row g is scaled by 1 / max |row g| over the cells
// sharing it.
#pragma once

#include <cublas_v2.h>
#include <cuda_runtime.h>
#include <cusolverDn.h>

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "../../include/ddhdg_b200.h"
#include "hdg_ndblas.cuh"

namespace ddhdg
{
  // A kernel's dynamic shared-memory limit is process-wide state.  It is set
  // once per device to the opt-in maximum (minus the kernel's static shared
  // memory) and never lowered, so that contexts launching one kernel with
  // different sizes from several host threads cannot race on it.
  inline cudaError_t
  allow_full_dynamic_smem(const void *fn)
  {
    static std::mutex                                  mu;
    static std::vector<std::pair<int, const void *>> done;
    int                                                dev = 0;
    cudaError_t                                        e   = cudaGetDevice(&dev);
    if (e != cudaSuccess)
      return e;
    std::lock_guard<std::mutex> lock(mu);
    for (auto &d : done)
      if (d.first == dev && d.second == fn)
        return cudaSuccess;
    cudaFuncAttributes fa;
    if ((e = cudaFuncGetAttributes(&fa, fn)) != cudaSuccess)
      return e;
    int optin = 0;
    if ((e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev)) != cudaSuccess)
      return e;
    if ((e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  optin - (int)fa.sharedSizeBytes)) != cudaSuccess)
      return e;
    done.push_back({dev, fn});
    return cudaSuccess;
  }

  struct NDAsm
  {
    int64_t off;     // front of the node (doubles)
    int64_t coff[2]; // fronts of the children
    int64_t moff[2]; // extend-add maps of the children
    int     cnF[2], cnE[2];
  };

  struct NDSol
  {
    int64_t off;  // front
    int64_t doff; // dof list
  };

  // rows of the leaf fronts: max |tt[a][:]| per global dof (bit pattern of a
  // non-negative double, so that an integer max is the double max)
  __global__ void
  nd_rowmax_kernel(int64_t ncells, int Nt, int nd, int F, const int64_t *cell_faces,
                   const double *tt, unsigned long long *dmax)
  {
    const int64_t tot = ncells * Nt;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < tot;
         idx += (int64_t)gridDim.x * blockDim.x)
      {
        const int64_t cell = idx / Nt;
        const int     a    = (int)(idx % Nt);
        const double *row  = tt + (cell * Nt + a) * (int64_t)Nt;
        double        m    = 0.;
        for (int b = 0; b < Nt; ++b)
          m = fmax(m, fabs(row[b]));
        const int64_t g = cell_faces[cell * F + a / nd] * nd + a % nd;
        atomicMax(dmax + g, (unsigned long long)__double_as_longlong(m));
      }
  }

  __global__ void
  nd_rowscale_kernel(int64_t n, const unsigned long long *dmax, double *dscale)
  {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
      {
        const double m = __longlong_as_double((long long)dmax[i]);
        dscale[i]      = (m > 0.) ? 1. / m : 1.;
      }
  }

  // leaf fronts (Nt x (Nt+1), column-major, last column the rhs) from the
  // condensed blocks; front order: faces on the physical boundary first
  // (local face order), then the others
  __global__ void
  nd_leaf_kernel(int64_t ncells, int Nt, int nd, int F, const uint8_t *pmask,
                 const int64_t *leaf_off, const int64_t *cell_faces, const double *tt,
                 const double *rhs, const int32_t *dflag, const double *dval,
                 const double *dscale, double *fronts)
  {
    for (int64_t cell = blockIdx.x; cell < ncells; cell += gridDim.x)
      {
        const unsigned msk = pmask[cell];
        int            rank[6];
        int            r = 0;
        for (int f = 0; f < F; ++f)
          if (msk & (1u << f))
            rank[f] = r++;
        for (int f = 0; f < F; ++f)
          if (!(msk & (1u << f)))
            rank[f] = r++;
        double        *Fr = fronts + leaf_off[cell];
        const double  *tc = tt + cell * (int64_t)Nt * Nt;
        const int32_t *fl = dflag + cell * (int64_t)Nt;
        for (int idx = threadIdx.x; idx < Nt * (Nt + 1); idx += blockDim.x)
          {
            const int     b  = idx / Nt, a = idx % Nt;
            const int     pa = rank[a / nd] * nd + a % nd;
            const int64_t g  = cell_faces[cell * F + a / nd] * nd + a % nd;
            if (b < Nt)
              {
                const int pb = rank[b / nd] * nd + b % nd;
                Fr[(int64_t)pb * Nt + pa] =
                  fl[a] ? (a == b ? 1. : 0.) : tc[(int64_t)a * Nt + b] * dscale[g];
              }
            else
              Fr[(int64_t)Nt * Nt + pa] = fl[a] ? dval[cell * Nt + a] : rhs[cell * Nt + a] * dscale[g];
          }
      }
  }

  // extend-add of child s's Schur complement (kept rows/columns and the rhs
  // column) into the node's front: CTA (node, range of `per` elements, at
  // least NDAsmElems, of the child's (cnK + 1) x cnK block, column-major),
  // one element per thread and step, so that the reads are coalesced over
  // the child's rows and every thread has work even for the few kept dofs of
  // the low fronts.
  // The two children are added by two launches, one after the other (they
  // overlap on the split-plane block).
  constexpr int NDAsmElems = 2048;

  __global__ void
  nd_assemble_kernel(int nF, int s, int64_t per, const NDAsm *nodes, const int32_t *emap, double *fronts)
  {
    const NDAsm    nd  = nodes[blockIdx.x];
    const int      cnF = nd.cnF[s], cnE = nd.cnE[s], cnK = cnF - cnE;
    const int64_t  tot = (int64_t)(cnK + 1) * cnK;
    const int64_t  e0  = (int64_t)blockIdx.y * per;
    if (e0 >= tot)
      return;
    const int64_t  e1  = e0 + per < tot ? e0 + per : tot;
    double        *Fv  = fronts + nd.off;
    const double  *Fc  = fronts + nd.coff[s];
    const int32_t *map = emap + nd.moff[s];
    for (int64_t e = e0 + threadIdx.x; e < e1; e += blockDim.x)
      {
        const int j  = (int)(e / cnK), i = (int)(e - (int64_t)j * cnK);
        const int pj = (j < cnK) ? map[j] : nF;
        Fv[(int64_t)pj * nF + map[i]] += Fc[(int64_t)(cnE + j) * cnF + cnE + i];
      }
  }

  // x_E = y_E - W x_K for every node of a batch.  CTA (node, block of R
  // eliminated rows) of R x S threads: thread (row t % R, slice t / R) sums
  // the terms k = slice, slice + S, ... of W x_K (for one k the R rows are
  // consecutive in memory), and the S partial sums of a row are added in
  // shared memory.  Short dependency chains: the top fronts have few rows per
  // node and thousands of kept dofs.
  __global__ void
  nd_backsolve_kernel(int nF, int nE, int R, const NDSol *nodes, const int32_t *fdofs,
                      const double *fronts, double *x)
  {
    extern __shared__ double sh[];
    const NDSol    n    = nodes[blockIdx.x];
    const int      nK   = nF - nE;
    const int      S    = blockDim.x / R;
    double        *xk   = sh;
    double        *part = sh + nK;
    const int32_t *dl   = fdofs + n.doff;
    for (int k = threadIdx.x; k < nK; k += blockDim.x)
      xk[k] = x[dl[nE + k]];
    __syncthreads();
    const double *Fv = fronts + n.off;
    const int     t  = threadIdx.x, il = t % R, sl = t / R;
    const int     i  = blockIdx.y * R + il;
    if (sl < S)
      {
        double v = 0.;
        if (i < nE)
          for (int k = sl; k < nK; k += S)
            v += Fv[(int64_t)(nE + k) * nF + i] * xk[k];
        part[sl * R + il] = v;
      }
    __syncthreads();
    if (t < R && i < nE)
      {
        double v = Fv[(int64_t)nF * nF + i];
        for (int q = 0; q < S; ++q)
          v -= part[q * R + t];
        x[dl[i]] = v;
      }
  }

  // rows per CTA and slices of the kept dofs of the back substitution of a
  // batch (R x S <= 1024 threads, about 8 or more terms per thread)
  inline void
  nd_backsolve_shape(int nE, int nK, int &R, int &S)
  {
    R = nE < 32 ? nE : 32;
    S = (nK + 7) / 8;
    S = S < 1 ? 1 : S;
    S = S > 1024 / R ? 1024 / R : S;
  }

  // row permutation of a batch's LU factorisations: the sequential swaps of
  // ipiv (1-based) turned into perm[i] = source row of row i; one thread per
  // front
  __global__ void
  nd_pivperm_kernel(int nb, int nE, const int *ipiv, int *perm)
  {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nb)
      return;
    const int *pv = ipiv + (int64_t)q * nE;
    int       *pm = perm + (int64_t)q * nE;
    for (int i = 0; i < nE; ++i)
      pm[i] = i;
    for (int j = 0; j < nE; ++j)
      {
        const int k = pv[j] - 1;
        const int t = pm[j];
        pm[j]       = pm[k];
        pm[k]       = t;
      }
  }

  // B = P B for the rows 0..nE-1 of the columns [nE, nF] of every front of a
  // batch (the right-hand sides of F_EE W = [F_EK | r_E]), in place, one
  // column at a time through shared memory; CTA (front, block of columns)
  constexpr int NDPermCols = 8;

  __global__ void
  nd_rowperm_kernel(int nE, int nF, const NDSol *nodes, const int *perm, double *fronts)
  {
    extern __shared__ double col[];
    const int64_t off = nodes[blockIdx.x].off;
    const int    *pm  = perm + (int64_t)blockIdx.x * nE;
    const int     c0  = blockIdx.y * NDPermCols;
    const int     c1  = min(nF - nE + 1, c0 + NDPermCols);
    for (int c = c0; c < c1; ++c)
      {
        double *B = fronts + off + (int64_t)(nE + c) * nF;
        for (int i = threadIdx.x; i < nE; i += blockDim.x)
          col[i] = B[i];
        __syncthreads();
        for (int i = threadIdx.x; i < nE; i += blockDim.x)
          B[i] = col[pm[i]];
        __syncthreads();
      }
  }

  // Small fronts (nE <= NDSmallE): the whole elimination of a front in one
  // CTA.  F_EE and [F_EK | r_E] are staged in shared memory; LU with partial
  // pivoting (row swaps in shared memory), back substitution to
  // W = F_EE^-1 [F_EK | r_E] (written back to the front for the downward
  // pass), then F_KK -= F_KE W in global memory with 4 x 4 register tiles
  // (F_KE read from the front, coalesced over rows).  info[front] = first
  // zero pivot (1-based) or 0.  Two launch forms of the same body: without a
  // register cap (the 36-dof fronts), and capped for MINB CTAs per SM (the
  // smallest fronts of the lowest levels gain from 4 or 5).
  constexpr int NDSmallE = 36;

  __device__ __forceinline__ void
  nd_small_front(int nE, int nK, const NDSol *nodes, int *info, double *fronts)
  {
    extern __shared__ double sm[];
    __shared__ int     piv_s, sing_s;
    const int          nF = nE + nK, nc = nK + 1;
    double            *A  = sm;              // [nE][nE]  column-major
    double            *B  = A + nE * nE;     // [nE][nc]  column-major
    double            *Fv = fronts + nodes[blockIdx.x].off;
    const int          tid = threadIdx.x, T = blockDim.x;
    for (int idx = tid; idx < nE * nE; idx += T)
      A[idx] = Fv[(int64_t)(idx / nE) * nF + idx % nE];
    for (int idx = tid; idx < nE * nc; idx += T)
      B[idx] = Fv[(int64_t)(nE + idx / nE) * nF + idx % nE];
    if (tid == 0)
      sing_s = 0;
    __syncthreads();
    for (int j = 0; j < nE; ++j)
      {
        if (tid < 32)
          {
            double best = -1.;
            int    bi   = nE;
            for (int i = j + tid; i < nE; i += 32)
              {
                const double v = fabs(A[i + j * nE]);
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
            if (tid == 0)
              {
                piv_s = (bi < nE) ? bi : j;
                if (!(best > 0.) || !isfinite(best))
                  if (sing_s == 0)
                    sing_s = j + 1;
              }
          }
        __syncthreads();
        const int p = piv_s;
        if (p != j)
          for (int c = tid; c < nE + nc; c += T)
            {
              double *X = (c < nE) ? A + c * nE : B + (c - nE) * nE;
              const double t = X[j];
              X[j]           = X[p];
              X[p]           = t;
            }
        __syncthreads();
        const double d  = A[j + j * nE];
        const double hr = (d != 0.) ? 1. / d : 0.;
        for (int i = j + 1 + tid; i < nE; i += T)
          A[i + j * nE] *= hr;
        __syncthreads();
        const int nr = nE - j - 1;
        if (nr > 0)
          for (int idx = tid; idx < nr * (nr + nc); idx += T)
            {
              const int i = j + 1 + idx % nr, c = idx / nr;
              double   *X = (c < nr) ? A + (j + 1 + c) * nE : B + (c - nr) * nE;
              X[i] -= A[i + j * nE] * X[j];
            }
        __syncthreads();
      }
    // back substitution with U
    for (int j = nE - 1; j >= 0; --j)
      {
        const double d  = A[j + j * nE];
        const double hr = (d != 0.) ? 1. / d : 0.;
        for (int c = tid; c < nc; c += T)
          B[j + c * nE] *= hr;
        __syncthreads();
        if (j > 0)
          for (int idx = tid; idx < j * nc; idx += T)
            {
              const int i = idx % j, c = idx / j;
              B[i + c * nE] -= A[i + j * nE] * B[j + c * nE];
            }
        __syncthreads();
      }
    for (int idx = tid; idx < nE * nc; idx += T)
      Fv[(int64_t)(nE + idx / nE) * nF + idx % nE] = B[idx];
    // Schur update of the kept block and the kept rhs: thread tile of rows
    // i0 + r nrt (r < 4, consecutive threads take consecutive rows) and
    // columns c0 .. c0 + 3
    {
      constexpr int RT = 4, CT = 4;
      const int     nrt = (nK + RT - 1) / RT, nct = (nc + CT - 1) / CT;
      for (int tile = tid; tile < nrt * nct; tile += T)
        {
          const int i0 = tile % nrt, c0 = (tile / nrt) * CT;
          double    acc[RT][CT];
#pragma unroll
          for (int r = 0; r < RT; ++r)
#pragma unroll
            for (int q = 0; q < CT; ++q)
              acc[r][q] = 0.;
          for (int k = 0; k < nE; ++k)
            {
              double cv[RT], bv[CT];
#pragma unroll
              for (int r = 0; r < RT; ++r)
                {
                  const int i = i0 + r * nrt;
                  cv[r]       = (i < nK) ? Fv[(int64_t)k * nF + nE + i] : 0.;
                }
#pragma unroll
              for (int q = 0; q < CT; ++q)
                bv[q] = (c0 + q < nc) ? B[k + (c0 + q) * nE] : 0.;
#pragma unroll
              for (int r = 0; r < RT; ++r)
#pragma unroll
                for (int q = 0; q < CT; ++q)
                  acc[r][q] += cv[r] * bv[q];
            }
#pragma unroll
          for (int r = 0; r < RT; ++r)
#pragma unroll
            for (int q = 0; q < CT; ++q)
              {
                const int i = i0 + r * nrt, c = c0 + q;
                if (i < nK && c < nc)
                  Fv[(int64_t)(nE + c) * nF + nE + i] -= acc[r][q];
              }
        }
    }
    if (tid == 0)
      info[blockIdx.x] = sing_s;
  }

  __global__ void
  nd_small_front_kernel(int nE, int nK, const NDSol *nodes, int *info, double *fronts)
  {
    nd_small_front(nE, nK, nodes, info, fronts);
  }

  template <int MINB>
  __global__ void __launch_bounds__(256, MINB)
  nd_small_front_capped_kernel(int nE, int nK, const NDSol *nodes, int *info, double *fronts)
  {
    nd_small_front(nE, nK, nodes, info, fronts);
  }

  // Dense LU with partial pivoting of F_EE for the fronts of a batch, one
  // CTA per front (NDLuTPB threads), all fronts of the batch at once; LAPACK
  // getrf output: L and U in place, ipiv (1-based sequential row swaps),
  // info = first zero pivot.  Right-looking, panels of NDLuNB columns:
  // - the panel (rows k0..nE-1) is factorised in shared memory: block-wide
  //   pivot search, row swap, and a row-owner update of the panel's columns;
  // - its swaps are applied to the rest of the front's rows in global
  //   memory (L2-resident), then U12 = L11^-1 A12 is solved column by column
  //   in registers by the thread that swapped the column;
  // - the trailing update A22 -= L21 U12 is a register-tiled FP64 product:
  //   a warp per group of 4 columns and 128-row block (a lane per row, rows
  //   32 apart), U12 staged in shared memory NDLuCols columns at a time.
  // For fronts of at most NDLuMaxE eliminated dofs (the panel fits in shared
  // memory).
  constexpr int NDLuNB   = 32;
  constexpr int NDLuCols = 64;
  constexpr int NDLuTPB  = 512;
  constexpr int NDLuMaxE = 576;

  __host__ __device__ inline size_t
  nd_lu_smem(int nE)
  {
    return ((size_t)nE * NDLuNB + (size_t)NDLuNB * NDLuCols) * sizeof(double);
  }

  __global__ void __launch_bounds__(NDLuTPB, 1)
  nd_lu_front_kernel(int nE, int nF, const NDSol *nodes, int *ipiv_all, int *info, double *fronts)
  {
    extern __shared__ double sm[];
    __shared__ double rv[NDLuTPB / 32];
    __shared__ int    ri[NDLuTPB / 32];
    __shared__ int    pv[NDLuNB];
    __shared__ int    sing_s;
    constexpr int     NW   = NDLuTPB / 32;
    const int         tid  = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    double           *A    = fronts + nodes[blockIdx.x].off; // F_EE: A[i + c nF]
    int              *ipiv = ipiv_all + (int64_t)blockIdx.x * nE;
    double           *Pn   = sm;                       // panel [NDLuNB][nE]: Pn[i + j nE]
    double           *Us   = sm + (size_t)nE * NDLuNB; // U12 chunk [NDLuNB][NDLuCols]
    if (tid == 0)
      sing_s = 0;
    for (int k0 = 0; k0 < nE; k0 += NDLuNB)
      {
        const int w = min(NDLuNB, nE - k0), m = nE - k0;
        for (int j = 0; j < w; ++j)
          for (int i = tid; i < m; i += NDLuTPB)
            Pn[i + j * nE] = A[(int64_t)(k0 + j) * nF + k0 + i];
        __syncthreads();
        // ---- panel factorisation
        for (int j = 0; j < w; ++j)
          {
            double best = -1.;
            int    bi   = m;
            for (int i = j + tid; i < m; i += NDLuTPB)
              {
                const double v = fabs(Pn[i + j * nE]);
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
            if (lane == 0)
              {
                rv[warp] = best;
                ri[warp] = bi;
              }
            __syncthreads();
            if (warp == 0)
              {
                best = lane < NW ? rv[lane] : -1.;
                bi   = lane < NW ? ri[lane] : m;
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
                if (lane == 0)
                  {
                    const int p  = (bi < m) ? bi : j;
                    pv[j]        = p;
                    ipiv[k0 + j] = k0 + p + 1;
                    if ((!(best > 0.) || !isfinite(best)) && sing_s == 0)
                      sing_s = k0 + j + 1;
                  }
              }
            __syncthreads();
            const int p = pv[j];
            if (p != j && tid < w)
              {
                const double t   = Pn[j + tid * nE];
                Pn[j + tid * nE] = Pn[p + tid * nE];
                Pn[p + tid * nE] = t;
              }
            __syncthreads();
            const double d  = Pn[j + j * nE];
            const double hr = (d != 0.) ? 1. / d : 0.;
            for (int i = j + 1 + tid; i < m; i += NDLuTPB)
              {
                const double l = Pn[i + j * nE] * hr;
                Pn[i + j * nE] = l;
                for (int c = j + 1; c < w; ++c)
                  Pn[i + c * nE] -= l * Pn[j + c * nE];
              }
            __syncthreads();
          }
        for (int j = 0; j < w; ++j)
          for (int i = tid; i < m; i += NDLuTPB)
            A[(int64_t)(k0 + j) * nF + k0 + i] = Pn[i + j * nE];
        // ---- the panel's swaps on the other columns; U12 for the trailing ones
        for (int c = tid; c < nE; c += NDLuTPB)
          {
            if (c >= k0 && c < k0 + w)
              continue;
            double *col = A + (int64_t)c * nF;
            for (int j = 0; j < w; ++j)
              {
                const int p = pv[j];
                if (p != j)
                  {
                    const double t = col[k0 + j];
                    col[k0 + j]    = col[k0 + p];
                    col[k0 + p]    = t;
                  }
              }
            if (c >= k0 + w)
              {
                double x[NDLuNB];
#pragma unroll
                for (int r = 0; r < NDLuNB; ++r)
                  x[r] = (r < w) ? col[k0 + r] : 0.;
#pragma unroll
                for (int r = 0; r < NDLuNB; ++r)
                  if (r < w)
#pragma unroll
                    for (int t = r + 1; t < NDLuNB; ++t)
                      if (t < w)
                        x[t] -= Pn[t + r * nE] * x[r];
#pragma unroll
                for (int r = 0; r < NDLuNB; ++r)
                  if (r < w)
                    col[k0 + r] = x[r];
              }
          }
        __syncthreads();
        // ---- trailing update A22 -= L21 U12
        const int r0 = k0 + w, nr = nE - r0;
        for (int cc = r0; cc < nE; cc += NDLuCols)
          {
            const int wc = min(NDLuCols, nE - cc);
            for (int idx = tid; idx < w * wc; idx += NDLuTPB)
              {
                const int t = idx % w, c = idx / w;
                Us[t * NDLuCols + c] = A[(int64_t)(cc + c) * nF + k0 + t];
              }
            __syncthreads();
            for (int g = warp; g < (wc + 3) / 4 * ((nr + 127) / 128); g += NW)
              {
                const int cg = g % ((wc + 3) / 4), rb = g / ((wc + 3) / 4);
                const int c0 = cg * 4;
                double    acc[4][4];
#pragma unroll
                for (int r = 0; r < 4; ++r)
#pragma unroll
                  for (int q = 0; q < 4; ++q)
                    acc[r][q] = 0.;
                for (int t = 0; t < w; ++t)
                  {
                    double lv[4], uv[4];
#pragma unroll
                    for (int r = 0; r < 4; ++r)
                      {
                        const int i = rb * 128 + lane + 32 * r; // row of A22
                        lv[r]       = (i < nr) ? Pn[(w + i) + t * nE] : 0.;
                      }
#pragma unroll
                    for (int q = 0; q < 4; ++q)
                      uv[q] = (c0 + q < wc) ? Us[t * NDLuCols + c0 + q] : 0.;
#pragma unroll
                    for (int r = 0; r < 4; ++r)
#pragma unroll
                      for (int q = 0; q < 4; ++q)
                        acc[r][q] += lv[r] * uv[q];
                  }
#pragma unroll
                for (int q = 0; q < 4; ++q)
                  if (c0 + q < wc)
#pragma unroll
                    for (int r = 0; r < 4; ++r)
                      {
                        const int i = rb * 128 + lane + 32 * r;
                        if (i < nr)
                          A[(int64_t)(cc + c0 + q) * nF + r0 + i] -= acc[r][q];
                      }
              }
            __syncthreads();
          }
      }
    if (tid == 0)
      info[blockIdx.x] = sing_s;
  }

  // Small fronts above the leaves, whole front in shared memory: the front
  // is assembled there from its two children's Schur complements (the
  // extend-add), eliminated there (LU with partial pivoting of F_EE,
  // W = F_EE^-1 [F_EK | r_E], F_KK -= F_KE W), and only its columns
  // nE..nF (W and the kept block with the kept rhs) are written to the
  // front in global memory: no zeroing of the front, no extend-add through
  // global memory, no second read.  One CTA per front; used where the front
  // (nF x (nF + 1) doubles) takes at most 100 KB of shared memory (two CTAs
  // per SM or more: with one, the 126-dof fronts ran slower than the
  // unfused path).
  __host__ __device__ inline size_t
  nd_fused_smem(int nF)
  {
    return (size_t)nF * (nF + 1) * sizeof(double);
  }

  __global__ void __launch_bounds__(256)
  nd_small_fused_kernel(int nE, int nK, const NDAsm *asmn, const int32_t *emap, int *info, double *fronts)
  {
    extern __shared__ double F[]; // [nF + 1 columns][nF rows], column-major
    __shared__ int     piv_s, sing_s;
    const int          nF = nE + nK, nc = nK + 1;
    const NDAsm        nd = asmn[blockIdx.x];
    const int          tid = threadIdx.x, T = blockDim.x;
    for (int idx = tid; idx < nF * (nF + 1); idx += T)
      F[idx] = 0.;
    if (tid == 0)
      sing_s = 0;
    __syncthreads();
    // extend-add of the two children (they overlap: one after the other)
    for (int s = 0; s < 2; ++s)
      {
        const int      cnF = nd.cnF[s], cnE = nd.cnE[s], cnK = cnF - cnE;
        const double  *Fc  = fronts + nd.coff[s];
        const int32_t *map = emap + nd.moff[s];
        const int      tot = (cnK + 1) * cnK;
        for (int e = tid; e < tot; e += T)
          {
            const int j = e / cnK, i = e - j * cnK;
            const int pj = (j < cnK) ? map[j] : nF;
            F[pj * nF + map[i]] += Fc[(int64_t)(cnE + j) * cnF + cnE + i];
          }
        __syncthreads();
      }
    // LU of F_EE with the row swaps and updates carried across all columns
    for (int j = 0; j < nE; ++j)
      {
        if (tid < 32)
          {
            double best = -1.;
            int    bi   = nE;
            for (int i = j + tid; i < nE; i += 32)
              {
                const double v = fabs(F[i + j * nF]);
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
            if (tid == 0)
              {
                piv_s = (bi < nE) ? bi : j;
                if ((!(best > 0.) || !isfinite(best)) && sing_s == 0)
                  sing_s = j + 1;
              }
          }
        __syncthreads();
        const int p = piv_s;
        if (p != j)
          for (int c = tid; c <= nF; c += T)
            {
              const double t = F[j + c * nF];
              F[j + c * nF]  = F[p + c * nF];
              F[p + c * nF]  = t;
            }
        __syncthreads();
        const double d  = F[j + j * nF];
        const double hr = (d != 0.) ? 1. / d : 0.;
        for (int i = j + 1 + tid; i < nE; i += T)
          F[i + j * nF] *= hr;
        __syncthreads();
        const int nr = nE - j - 1;
        if (nr > 0)
          for (int idx = tid; idx < nr * (nF - j); idx += T)
            {
              const int i = j + 1 + idx % nr, c = j + 1 + idx / nr;
              F[i + c * nF] -= F[i + j * nF] * F[j + c * nF];
            }
        __syncthreads();
      }
    // back substitution with U on the columns nE..nF (W)
    for (int j = nE - 1; j >= 0; --j)
      {
        const double d  = F[j + j * nF];
        const double hr = (d != 0.) ? 1. / d : 0.;
        for (int c = nE + tid; c <= nF; c += T)
          F[j + c * nF] *= hr;
        __syncthreads();
        if (j > 0)
          for (int idx = tid; idx < j * nc; idx += T)
            {
              const int i = idx % j, c = nE + idx / j;
              F[i + c * nF] -= F[i + j * nF] * F[j + c * nF];
            }
        __syncthreads();
      }
    // Schur update of the kept rows (F_KE and W are only read here)
    for (int idx = tid; idx < nK * nc; idx += T)
      {
        const int i = nE + idx % nK, c = nE + idx / nK;
        double    acc = 0.;
        for (int k = 0; k < nE; ++k)
          acc += F[i + k * nF] * F[k + c * nF];
        F[i + c * nF] -= acc;
      }
    __syncthreads();
    double *Fv = fronts + nd.off;
    for (int idx = tid; idx < nF * nc; idx += T)
      {
        const int i = idx % nF, c = nE + idx / nF;
        Fv[(int64_t)c * nF + i] = F[i + c * nF];
      }
    if (tid == 0)
      info[blockIdx.x] = sing_s;
  }

  // Mid fronts (NDSmallE < nE <= NDMidE), one CTA of 16 warps per front
  // (above 72 eliminated dofs the single-warp diagonal-block solves make it
  // slower than the batched cuBLAS path):
  // - LU of F_EE with partial pivoting in shared memory (row swaps in shared
  //   memory, the permutation kept as perm[i] = source row of row i);
  // - W = U^-1 L^-1 P [F_EK | r_E] in chunks of NDMidCols columns, staged in
  //   shared memory row-major (stride NDMidCols + 1: conflict-free by rows
  //   and by columns) with the permutation applied on the load: blocked
  //   triangular solves, each diagonal block of NDMidNB rows solved by one
  //   warp in registers (a lane per column), the rows beyond it updated by
  //   all warps (a warp per row, a lane per column);
  // - the chunk written back to the front over [F_EK | r_E].
  // The Schur update F_KK -= F_KE W follows as a batched GEMM.
  // info[front] = first zero pivot (1-based) or 0.
  constexpr int NDMidE    = 72;
  constexpr int NDMidCols = 32;
  constexpr int NDMidLdb  = NDMidCols + 1;
  constexpr int NDMidNB   = 16;
  constexpr int NDMidTPB  = 512;

  __host__ __device__ inline size_t
  nd_mid_smem(int nE)
  {
    return ((size_t)nE * nE + (size_t)nE * NDMidLdb + nE) * sizeof(double) + (size_t)nE * sizeof(int);
  }

  __global__ void __launch_bounds__(NDMidTPB)
  nd_mid_front_kernel(int nE, int nK, const NDSol *nodes, int *info, double *fronts)
  {
    extern __shared__ double sm[];
    __shared__ int     piv_s, sing_s;
    constexpr int      NW = NDMidTPB / 32;
    const int          nF = nE + nK, nc = nK + 1;
    double            *A    = sm;                // [nE][nE] column-major
    double            *Bc   = A + nE * nE;       // [nE][NDMidLdb] row-major
    double            *dinv = Bc + nE * NDMidLdb;
    int               *perm = reinterpret_cast<int *>(dinv + nE);
    double            *Fv   = fronts + nodes[blockIdx.x].off;
    const int          tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int c = warp; c < nE; c += NW)
      for (int i = lane; i < nE; i += 32)
        A[i + c * nE] = Fv[(int64_t)c * nF + i];
    for (int i = tid; i < nE; i += NDMidTPB)
      perm[i] = i;
    if (tid == 0)
      sing_s = 0;
    __syncthreads();
    // ------------------------------------------------------------ LU of F_EE
    for (int j = 0; j < nE; ++j)
      {
        if (warp == 0)
          {
            double best = -1.;
            int    bi   = nE;
            for (int i = j + lane; i < nE; i += 32)
              {
                const double v = fabs(A[i + j * nE]);
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
            if (lane == 0)
              {
                const int p = (bi < nE) ? bi : j;
                piv_s       = p;
                const int t = perm[j];
                perm[j]     = perm[p];
                perm[p]     = t;
                if (!(best > 0.) || !isfinite(best))
                  if (sing_s == 0)
                    sing_s = j + 1;
              }
          }
        __syncthreads();
        const int p = piv_s;
        if (p != j)
          for (int c = tid; c < nE; c += NDMidTPB)
            {
              const double t = A[j + c * nE];
              A[j + c * nE]  = A[p + c * nE];
              A[p + c * nE]  = t;
            }
        __syncthreads();
        const double d  = A[j + j * nE];
        const double hr = (d != 0.) ? 1. / d : 0.;
        if (tid == 0)
          dinv[j] = hr;
        for (int i = j + 1 + tid; i < nE; i += NDMidTPB)
          A[i + j * nE] *= hr;
        __syncthreads();
        for (int c = j + 1 + warp; c < nE; c += NW)
          {
            const double ajc = A[j + c * nE];
            for (int i = j + 1 + lane; i < nE; i += 32)
              A[i + c * nE] -= A[i + j * nE] * ajc;
          }
        __syncthreads();
      }
    // ------------------------------------------- W, NDMidCols columns at a time
    const int nblk = (nE + NDMidNB - 1) / NDMidNB;
    for (int c0 = 0; c0 < nc; c0 += NDMidCols)
      {
        const int w = min(NDMidCols, nc - c0);
        for (int c = warp; c < w; c += NW)
          for (int i = lane; i < nE; i += 32)
            Bc[i * NDMidLdb + c] = Fv[(int64_t)(nE + c0 + c) * nF + perm[i]];
        __syncthreads();
        // unit lower triangle, block by block
        for (int kb = 0; kb < nE; kb += NDMidNB)
          {
            const int kn = min(NDMidNB, nE - kb);
            if (warp == 0 && lane < w)
              {
                double x[NDMidNB];
#pragma unroll
                for (int r = 0; r < NDMidNB; ++r)
                  x[r] = (r < kn) ? Bc[(kb + r) * NDMidLdb + lane] : 0.;
#pragma unroll
                for (int r = 0; r < NDMidNB; ++r)
#pragma unroll
                  for (int q = r + 1; q < NDMidNB; ++q)
                    if (q < kn)
                      x[q] -= A[(kb + q) + (kb + r) * nE] * x[r];
#pragma unroll
                for (int r = 0; r < NDMidNB; ++r)
                  if (r < kn)
                    Bc[(kb + r) * NDMidLdb + lane] = x[r];
              }
            __syncthreads();
            if (kb + kn < nE && lane < w)
              {
                double x[NDMidNB];
#pragma unroll
                for (int r = 0; r < NDMidNB; ++r)
                  x[r] = (r < kn) ? Bc[(kb + r) * NDMidLdb + lane] : 0.;
                for (int i = kb + kn + warp; i < nE; i += NW)
                  {
                    double acc = 0.;
#pragma unroll
                    for (int r = 0; r < NDMidNB; ++r)
                      if (r < kn)
                        acc += A[i + (kb + r) * nE] * x[r];
                    Bc[i * NDMidLdb + lane] -= acc;
                  }
              }
            __syncthreads();
          }
        // upper triangle, block by block from the last
        for (int bq = nblk - 1; bq >= 0; --bq)
          {
            const int kb = bq * NDMidNB;
            const int kn = min(NDMidNB, nE - kb);
            if (warp == 0 && lane < w)
              {
                double x[NDMidNB];
#pragma unroll
                for (int r = 0; r < NDMidNB; ++r)
                  x[r] = (r < kn) ? Bc[(kb + r) * NDMidLdb + lane] : 0.;
#pragma unroll
                for (int r = NDMidNB - 1; r >= 0; --r)
                  if (r < kn)
                    {
                      x[r] *= dinv[kb + r];
#pragma unroll
                      for (int q = 0; q < r; ++q)
                        x[q] -= A[(kb + q) + (kb + r) * nE] * x[r];
                    }
#pragma unroll
                for (int r = 0; r < NDMidNB; ++r)
                  if (r < kn)
                    Bc[(kb + r) * NDMidLdb + lane] = x[r];
              }
            __syncthreads();
            if (kb > 0 && lane < w)
              {
                double x[NDMidNB];
#pragma unroll
                for (int r = 0; r < NDMidNB; ++r)
                  x[r] = (r < kn) ? Bc[(kb + r) * NDMidLdb + lane] : 0.;
                for (int i = warp; i < kb; i += NW)
                  {
                    double acc = 0.;
#pragma unroll
                    for (int r = 0; r < NDMidNB; ++r)
                      if (r < kn)
                        acc += A[i + (kb + r) * nE] * x[r];
                    Bc[i * NDMidLdb + lane] -= acc;
                  }
              }
            __syncthreads();
          }
        for (int c = warp; c < w; c += NW)
          for (int i = lane; i < nE; i += 32)
            Fv[(int64_t)(nE + c0 + c) * nF + i] = Bc[i * NDMidLdb + c];
        __syncthreads();
      }
    if (tid == 0)
      info[blockIdx.x] = sing_s;
  }

  // -------------------------------------------------------------- host side
  class NDSolver
  {
  public:
    struct Mesh
    {
      int     dim            = 2;
      int     n[3]           = {1, 1, 1};
      int64_t face_off[3]    = {0, 0, 0};
      int     face_ext[3][3] = {{1, 1, 1}, {1, 1, 1}, {1, 1, 1}};
      int64_t ncells = 0, nfaces = 0;
      int     F  = 4;
      int     nd = 1; // trace dofs per face (enabled components x face nodes)
    };

    ~NDSolver() { release(); }

    bool built() const { return built_; }

    int64_t front_bytes() const { return front_total_ * (int64_t)sizeof(double); }

    // Device bytes that build() allocates for the planned mesh: fronts,
    // pivots, inverted diagonal blocks, the maps and the scaling vectors,
    // each allocation rounded up to the allocator's 2 MiB granularity, a
    // bound of 64 nE doubles per side stream for the LU workspace of the
    // largest front (the library reports its size only once a handle
    // exists), and the library handles.  The caller's plan() must have
    // succeeded.
    // side streams (each with its library handles) that the plan's large
    // fronts use: one per front of the largest per-front batch, at most NSide
    int
    side_count() const
    {
      int n = 0;
      for (const auto &bt : batches_)
        if (bt.big)
          n = std::max(n, (int)bt.nodes.size());
      return std::min(n, NSide);
    }

    int64_t
    planned_device_bytes() const
    {
      const int64_t g = (int64_t)2 << 20;
      int64_t       b = 0;
      auto          add = [&](int64_t bytes) { b += (std::max<int64_t>(bytes, 16) + g - 1) / g * g; };
      add(front_total_ * 8);
      add(std::max<int64_t>(piv_total_, 1) * 4);
      add(std::max<int64_t>(piv_total_, 1) * 4);
      add(((int64_t)nodes_.size() + 1) * 4);
      int64_t tinv = 1, big_nE = 1;
      for (const auto &bt : batches_)
        {
          if (bt.nE > 0 && !bt.small && !bt.fused && !bt.mid)
            tinv = std::max<int64_t>(tinv, (int64_t)bt.nodes.size() * ((bt.nE + NDTB - 1) / NDTB) * 2 * NDTB * NDTB);
          if (bt.big)
            big_nE = std::max<int64_t>(big_nE, bt.nE);
        }
      add(tinv * 8);
      add((int64_t)fdofs_h_.size() * 4);
      add((int64_t)emap_h_.size() * 4);
      add((int64_t)leaf_off_h_.size() * 8);
      add((int64_t)pmask_h_.size());
      add((int64_t)cell_faces_.size() * 8);
      add((int64_t)asm_h_.size() * (int64_t)sizeof(NDAsm));
      add((int64_t)sol_h_.size() * (int64_t)sizeof(NDSol));
      add((int64_t)ptr_h_.size() * 8);
      const int64_t ndofs = M_.nfaces * (int64_t)M_.nd;
      add(ndofs * 8);
      add(ndofs * 8);
      add((int64_t)side_count() * 64 * big_nE * 8);
      // library handles: one cuBLAS handle, and a cuBLAS and a cuSOLVER
      // handle per side stream (measured on CUDA 12.9: about 70 MB and
      // 300 MB of device memory each)
      b += (int64_t)(1 + side_count()) * (80 << 20) + (int64_t)side_count() * (320 << 20);
      return b;
    }

    // the plan's batches: {height, eliminated dofs, kept dofs, fronts, kind}
    // with kind 0 fused, 1 small, 2 mid, 3 own LU + batched products, 4 big
    std::vector<std::vector<int>>
    batch_shapes() const
    {
      std::vector<std::vector<int>> out;
      for (const auto &b : batches_)
        out.push_back({b.height, b.nE, b.nK, (int)b.nodes.size(),
                       b.fused ? 0 : b.small ? 1 : b.mid ? 2 : b.big ? 4 : 3});
      return out;
    }

    // symbolic phase on the host: tree, fronts, maps and batches.  The plan
    // depends on the mesh shape only, so plans are kept in a small process-
    // wide cache: contexts of the same shape (the serving layer's requests,
    // a bias sweep's solvers) reuse it instead of building it again (0.5 s
    // on the host for 65 536 cells).
    int
    plan(const Mesh &M, std::string &err)
    {
      release();
      {
        std::lock_guard<std::mutex> lock(plan_cache_mutex());
        for (auto &e : plan_cache())
          if (same_mesh(e->M, M))
            {
              load_plan(*e);
              return DDHDG_OK;
            }
      }
      int r = plan_uncached(M, err);
      if (r)
        return r;
      std::shared_ptr<PlanState> e(new PlanState);
      save_plan(*e);
      std::lock_guard<std::mutex> lock(plan_cache_mutex());
      auto &c = plan_cache();
      c.insert(c.begin(), std::move(e));
      // at most 32 plans (two modes of 16 requests in flight), and no more
      // than 4 GB of host copies
      size_t bytes = 0, keep = 0;
      for (; keep < c.size() && keep < 32; ++keep)
        {
          bytes += c[keep]->bytes();
          if (bytes > ((size_t)4 << 30) && keep > 0)
            break;
        }
      c.resize(keep);
      return DDHDG_OK;
    }

  private:
    struct PlanState;
    static bool
    same_mesh(const Mesh &a, const Mesh &b)
    {
      if (a.dim != b.dim || a.ncells != b.ncells || a.nfaces != b.nfaces || a.F != b.F || a.nd != b.nd)
        return false;
      for (int i = 0; i < 3; ++i)
        {
          if (a.n[i] != b.n[i] || a.face_off[i] != b.face_off[i])
            return false;
          for (int j = 0; j < 3; ++j)
            if (a.face_ext[i][j] != b.face_ext[i][j])
              return false;
        }
      return true;
    }
    static std::mutex &
    plan_cache_mutex()
    {
      static std::mutex mu;
      return mu;
    }
    static std::vector<std::shared_ptr<PlanState>> &
    plan_cache()
    {
      static std::vector<std::shared_ptr<PlanState>> c;
      return c;
    }

  public:
    int
    plan_uncached(const Mesh &M, std::string &err)
    {
      M_ = M;
      if (M.F > 6 || M.dim < 1 || M.dim > 3)
        return bad(err, "unsupported mesh for the nested-dissection solve");
      if (M.nfaces * (int64_t)M.nd > INT32_MAX)
        return bad(err, "too many trace dofs for 32-bit dof lists");
      cell_faces_.assign(M.ncells * M.F, 0);
      for (int64_t c = 0; c < M.ncells; ++c)
        for (int f = 0; f < M.F; ++f)
          cell_faces_[c * M.F + f] = face_of_cell(c, f);
      nodes_.clear();
      int lo[3] = {0, 0, 0}, hi[3] = {M.n[0], M.dim > 1 ? M.n[1] : 1, M.dim > 2 ? M.n[2] : 1};
      root_ = make_node(lo, hi);
      // batches: by height, then by shape
      int maxh = 0;
      for (auto &nd : nodes_)
        maxh = std::max(maxh, nd.height);
      std::vector<std::vector<int>> by_h(maxh + 1);
      for (int i = 0; i < (int)nodes_.size(); ++i)
        by_h[nodes_[i].height].push_back(i);
      batches_.clear();
      for (int h = 0; h <= maxh; ++h)
        {
          auto &ids = by_h[h];
          std::sort(ids.begin(), ids.end(), [this](int a, int b) {
            const auto &A = nodes_[a], &B = nodes_[b];
            if (A.nE != B.nE)
              return A.nE < B.nE;
            if (A.nK != B.nK)
              return A.nK < B.nK;
            return a < b;
          });
          for (size_t i = 0; i < ids.size();)
            {
              size_t j = i;
              while (j < ids.size() && nodes_[ids[j]].nE == nodes_[ids[i]].nE &&
                     nodes_[ids[j]].nK == nodes_[ids[i]].nK)
                ++j;
              Batch b;
              b.height = h;
              b.nE     = nodes_[ids[i]].nE;
              b.nK     = nodes_[ids[i]].nK;
              b.nodes.assign(ids.begin() + i, ids.begin() + j);
              batches_.push_back(std::move(b));
              i = j;
            }
        }
      // front, pivot and dof offsets in batch order
      int64_t off = 0, poff = 0, doff = 0;
      for (auto &b : batches_)
        {
          const int64_t nF = b.nE + b.nK;
          b.front_off      = off;
          b.piv_off        = poff;
          for (int id : b.nodes)
            {
              nodes_[id].off = off;
              off += nF * (nF + 1);
              nodes_[id].doff = doff;
              doff += nF;
            }
          poff += (int64_t)b.nE * b.nodes.size();
          b.front_end = off;
        }
      front_total_ = off;
      piv_total_   = poff;
      // dof lists and extend-add maps
      fdofs_h_.assign(doff, 0);
      for (auto &nd : nodes_)
        std::copy(nd.dofs.begin(), nd.dofs.end(), fdofs_h_.begin() + nd.doff);
      std::vector<int32_t> pos(M.nfaces * (int64_t)M.nd, -1);
      emap_h_.clear();
      for (auto &nd : nodes_)
        {
          if (nd.child[0] < 0)
            continue;
          for (int i = 0; i < (int)nd.dofs.size(); ++i)
            pos[nd.dofs[i]] = i;
          for (int s = 0; s < 2; ++s)
            {
              const auto &ch = nodes_[nd.child[s]];
              nd.moff[s]     = (int64_t)emap_h_.size();
              for (int k = ch.nE; k < (int)ch.dofs.size(); ++k)
                {
                  const int32_t p = pos[ch.dofs[k]];
                  if (p < 0)
                    return bad(err, "nested dissection: a kept dof is missing from the parent front");
                  emap_h_.push_back(p);
                }
            }
          for (int32_t g : nd.dofs)
            pos[g] = -1;
        }
      // leaves
      leaf_off_h_.assign(M.ncells, 0);
      pmask_h_.assign(M.ncells, 0);
      for (auto &nd : nodes_)
        if (nd.cell >= 0)
          {
            leaf_off_h_[nd.cell] = nd.off;
            pmask_h_[nd.cell]    = (uint8_t)nd.pmask;
          }
      // per-batch tables: extend-add, back substitution, pointer offsets
      asm_h_.clear();
      sol_h_.clear();
      ptr_h_.clear();
      max_nK_ = 0;
      for (auto &b : batches_)
        {
          const int nF = b.nE + b.nK;
          b.asm_off    = (int64_t)asm_h_.size();
          b.sol_off    = (int64_t)sol_h_.size();
          b.ptr_off    = (int64_t)ptr_h_.size();
          for (int id : b.nodes)
            {
              const auto &nd = nodes_[id];
              if (nd.child[0] >= 0)
                {
                  NDAsm a{};
                  a.off = nd.off;
                  for (int s = 0; s < 2; ++s)
                    {
                      const auto &ch = nodes_[nd.child[s]];
                      a.coff[s]      = ch.off;
                      a.moff[s]      = nd.moff[s];
                      a.cnF[s]       = ch.nE + ch.nK;
                      a.cnE[s]       = ch.nE;
                    }
                  asm_h_.push_back(a);
                  for (int s = 0; s < 2; ++s)
                    b.maxc[s] = std::max(b.maxc[s], a.cnF[s] - a.cnE[s] + 1);
                }
              sol_h_.push_back(NDSol{nd.off, nd.doff});
            }
          // F_EE, [F_EK | r_E], F_KE, F_KK of every node, as offsets
          for (int q = 0; q < 4; ++q)
            for (int id : b.nodes)
              {
                const int64_t o = nodes_[id].off;
                ptr_h_.push_back(q == 0   ? o
                                 : q == 1 ? o + (int64_t)b.nE * nF
                                 : q == 2 ? o + b.nE
                                          : o + (int64_t)b.nE * nF + b.nE);
              }
          b.big   = b.nE >= 384 && b.nodes.size() <= 32;
          b.small = !b.big && b.nE > 0 && b.nE <= NDSmallE && small_smem(b.nE, b.nK) <= 200 * 1024;
          b.mid   = !b.big && !b.small && b.nE > 0 && b.nE <= NDMidE && nd_mid_smem(b.nE) <= 220 * 1024;
          b.fused = b.small && b.height > 0 && nd_fused_smem(b.nE + b.nK) <= 100 * 1024;
          max_nK_ = std::max(max_nK_, b.nK);
        }
      return DDHDG_OK;
    }

    // symbolic phase (plan) and the device buffers
    int
    build(const Mesh &M, std::string &err)
    {
      int r;
      if ((r = plan(M, err)))
        return r;
      if ((r = dmalloc(d_fronts_, front_total_ * sizeof(double), err)) ||
          (r = dmalloc(d_piv_, std::max<int64_t>(piv_total_, 1) * sizeof(int), err)) ||
          (r = dmalloc(d_perm_, std::max<int64_t>(piv_total_, 1) * sizeof(int), err)))
        return r;
      // one info per node, plus a sink for the solves' parameter status
      if ((r = dmalloc(d_info_, (nodes_.size() + 1) * sizeof(int), err)))
        return r;
      // inverted diagonal blocks of the triangular solves (largest batch)
      {
        int64_t tinv = 1;
        for (const auto &b : batches_)
          if (b.nE > 0 && !b.small && !b.fused && !b.mid)
            tinv = std::max<int64_t>(tinv, (int64_t)b.nodes.size() * ((b.nE + NDTB - 1) / NDTB) * 2 * NDTB * NDTB);
        if ((r = dmalloc(d_tinv_, tinv * sizeof(double), err)))
          return r;
        const char *e = getenv("DDHDG_ND_OWN_TRSM");
        own_trsm_     = e && e[0] == '1';
        const char *g = getenv("DDHDG_ND_OWN_GEMM");
        own_gemm_     = g && g[0] == '1';
      }
      if ((r = upload(d_fdofs_, fdofs_h_, err)) || (r = upload(d_emap_, emap_h_, err)) ||
          (r = upload(d_leaf_off_, leaf_off_h_, err)) || (r = upload(d_pmask_, pmask_h_, err)) ||
          (r = upload(d_cell_faces_, cell_faces_, err)) || (r = upload(d_asm_, asm_h_, err)) ||
          (r = upload(d_sol_, sol_h_, err)))
        return r;
      std::vector<double *> ptrs(ptr_h_.size());
      for (size_t q = 0; q < ptr_h_.size(); ++q)
        ptrs[q] = d_fronts_ + ptr_h_[q];
      if ((r = upload(d_ptr_, ptrs, err)))
        return r;
      const int64_t ndofs = M.nfaces * (int64_t)M.nd;
      if ((r = dmalloc(d_dmax_, ndofs * sizeof(unsigned long long), err)) ||
          (r = dmalloc(d_dscale_, ndofs * sizeof(double), err)))
        return r;
      if (cublasCreate(&blas_) != CUBLAS_STATUS_SUCCESS)
        return bad(err, "cublasCreate failed", DDHDG_SOLVER_ERROR);
      // side streams with their own handles, only as many as the largest
      // per-front batch uses (a cuSOLVER handle holds about 300 MB of device
      // memory, a cuBLAS one about 70 MB)
      nside_ = side_count();
      if (cudaEventCreateWithFlags(&ev_fork_, cudaEventDisableTiming) != cudaSuccess)
        return bad(err, "cudaEventCreate failed", DDHDG_CUDA_ERROR);
      if (cudaStreamCreateWithFlags(&cap_, cudaStreamNonBlocking) != cudaSuccess)
        return bad(err, "cudaStreamCreate failed", DDHDG_CUDA_ERROR);
      for (int k = 0; k < nside_; ++k)
        {
          if (cudaStreamCreateWithFlags(&side_[k], cudaStreamNonBlocking) != cudaSuccess ||
              cudaEventCreateWithFlags(&ev_join_[k], cudaEventDisableTiming) != cudaSuccess)
            return bad(err, "cudaStreamCreate failed", DDHDG_CUDA_ERROR);
          if (cublasCreate(&side_blas_[k]) != CUBLAS_STATUS_SUCCESS ||
              cusolverDnCreate(&side_dn_[k]) != CUSOLVER_STATUS_SUCCESS)
            return bad(err, "handle creation failed", DDHDG_SOLVER_ERROR);
          cublasSetStream(side_blas_[k], side_[k]);
          cusolverDnSetStream(side_dn_[k], side_[k]);
        }
      int64_t big_ws = 0;
      for (auto &b : batches_)
        if (b.big)
          for (int id : b.nodes)
            {
              int       lw = 0;
              const int nF = b.nE + b.nK;
              if (cusolverDnDgetrf_bufferSize(side_dn_[0], b.nE, b.nE, d_fronts_ + nodes_[id].off, nF, &lw) !=
                  CUSOLVER_STATUS_SUCCESS)
                return bad(err, "cusolverDnDgetrf_bufferSize failed", DDHDG_SOLVER_ERROR);
              big_ws = std::max<int64_t>(big_ws, lw);
            }
      work_per_ = std::max<int64_t>(big_ws, 1);
      if ((r = dmalloc(d_work_, std::max(nside_, 1) * work_per_ * sizeof(double), err)))
        return r;
      if (allow_full_dynamic_smem(reinterpret_cast<const void *>(nd_small_front_kernel)) != cudaSuccess ||
          allow_full_dynamic_smem(reinterpret_cast<const void *>(nd_small_front_capped_kernel<4>)) != cudaSuccess ||
          allow_full_dynamic_smem(reinterpret_cast<const void *>(nd_small_front_capped_kernel<5>)) != cudaSuccess ||
          allow_full_dynamic_smem(reinterpret_cast<const void *>(nd_rowperm_kernel)) != cudaSuccess ||
          allow_full_dynamic_smem(reinterpret_cast<const void *>(nd_backsolve_kernel)) != cudaSuccess ||
          allow_full_dynamic_smem(reinterpret_cast<const void *>(nd_mid_front_kernel)) != cudaSuccess ||
          allow_full_dynamic_smem(reinterpret_cast<const void *>(nd_small_fused_kernel)) != cudaSuccess ||
          allow_full_dynamic_smem(reinterpret_cast<const void *>(nd_lu_front_kernel)) != cudaSuccess)
        return bad(err, "cannot raise the shared-memory limit of the trace-solve kernels", DDHDG_CUDA_ERROR);
      nodes_info_ = (int)nodes_.size();
      built_      = true;
      return DDHDG_OK;
    }

    // numeric phase: x (global trace dofs) from the per-cell condensed
    // blocks.  The whole sequence (about 10 launches per batch) is captured
    // in a CUDA graph on the second call with the same buffers and replayed
    // after that; the check for singular fronts stays outside the graph.
    // capture and replay of the numeric sequence on (default) or off
    void
    set_graphs(bool on)
    {
      use_graphs_ = on;
      if (!on && exec_)
        {
          cudaGraphExecDestroy(exec_);
          exec_ = nullptr;
        }
    }

    int
    solve(const double *tt, const double *rhs, const int32_t *dflag, const double *dval, int Nt,
          double *x, cudaStream_t s, int sm_count, std::string &err, bool check = true)
    {
      if (!built_)
        return bad(err, "nested-dissection solver not built");
      if (Nt != M_.F * M_.nd)
        return bad(err, "trace block size does not match the solver");
      const Key k{tt, rhs, dflag, dval, x, sm_count};
      int       r = DDHDG_OK;
      if (use_graphs_ && graphs_ok_ && exec_ && k == key_)
        {
          if (cudaGraphLaunch(exec_, s) != cudaSuccess)
            return bad(err, "cudaGraphLaunch failed", DDHDG_CUDA_ERROR);
        }
      else if (use_graphs_ && graphs_ok_ && k == key_ && !exec_)
        {
          // same buffers as the last (eager) call: capture, then launch
          cudaGraph_t gph = nullptr;
          if (cudaStreamBeginCapture(cap_, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
            {
              cudaGetLastError();
              graphs_ok_ = false;
              r          = enqueue(tt, rhs, dflag, dval, Nt, x, s, sm_count, err);
            }
          else
            {
              const int         rc = enqueue(tt, rhs, dflag, dval, Nt, x, cap_, sm_count, err);
              const cudaError_t e  = cudaStreamEndCapture(cap_, &gph);
              if (rc || e != cudaSuccess || !gph ||
                  cudaGraphInstantiate(&exec_, gph, 0) != cudaSuccess)
                {
                  cudaGetLastError();
                  exec_      = nullptr;
                  graphs_ok_ = false; // this build cannot capture: stay eager
                  r          = enqueue(tt, rhs, dflag, dval, Nt, x, s, sm_count, err);
                }
              else if (cudaGraphLaunch(exec_, s) != cudaSuccess)
                r = bad(err, "cudaGraphLaunch failed", DDHDG_CUDA_ERROR);
              if (gph)
                cudaGraphDestroy(gph);
            }
        }
      else
        {
          if (exec_)
            cudaGraphExecDestroy(exec_);
          exec_ = nullptr;
          key_  = k;
          r     = enqueue(tt, rhs, dflag, dval, Nt, x, s, sm_count, err);
        }
      if (r)
        return r;
      // check = false: the caller reads the per-front pivot status later
      // (check_info), so that solves on several streams overlap
      return check ? check_info(s, err) : DDHDG_OK;
    }

  private:
    struct Key
    {
      const void *tt, *rhs, *dflag, *dval, *x;
      int         sm;
      bool
      operator==(const Key &o) const
      {
        return tt == o.tt && rhs == o.rhs && dflag == o.dflag && dval == o.dval && x == o.x && sm == o.sm;
      }
    };

    // the numeric phase's launches on stream s (no host synchronisation)
    int
    enqueue(const double *tt, const double *rhs, const int32_t *dflag, const double *dval, int Nt,
            double *x, cudaStream_t s, int sm_count, std::string &err)
    {
      const auto   &M     = M_;
      const int64_t ndofs = M.nfaces * (int64_t)M.nd;
      const int     grid  = sm_count * 8;
      cublasSetStream(blas_, s);
      // row equilibration
      if (cudaMemsetAsync(d_dmax_, 0, ndofs * sizeof(unsigned long long), s) != cudaSuccess)
        return bad(err, "memset failed", DDHDG_CUDA_ERROR);
      nd_rowmax_kernel<<<grid, 256, 0, s>>>(M.ncells, Nt, M.nd, M.F, d_cell_faces_, tt, d_dmax_);
      nd_rowscale_kernel<<<grid, 256, 0, s>>>(ndofs, d_dmax_, d_dscale_);
      // leaves
      nd_leaf_kernel<<<grid, 256, 0, s>>>(M.ncells, Nt, M.nd, M.F, d_pmask_, d_leaf_off_,
                                          d_cell_faces_, tt, rhs, dflag, dval, d_dscale_, d_fronts_);
      if (cudaMemsetAsync(d_info_, 0, (nodes_info_ + 1) * sizeof(int), s) != cudaSuccess)
        return bad(err, "memset failed", DDHDG_CUDA_ERROR);
      // upward pass
      int info_base = 0;
      for (auto &b : batches_)
        {
          const int nF = b.nE + b.nK;
          const int nb = (int)b.nodes.size();
          if (b.height > 0 && !b.fused)
            {
              if (cudaMemsetAsync(d_fronts_ + b.front_off, 0,
                                  (b.front_end - b.front_off) * sizeof(double), s) != cudaSuccess)
                return bad(err, "memset failed", DDHDG_CUDA_ERROR);
              for (int c = 0; c < 2; ++c)
                {
                  const int64_t ck = b.maxc[c] - 1; // largest child nK of this pass
                  if (ck <= 0)
                    continue;
                  const int64_t tot = (ck + 1) * ck;
                  const int64_t per = std::max<int64_t>(NDAsmElems, (tot + 65534) / 65535);
                  const dim3    g2(nb, (unsigned)((tot + per - 1) / per));
                  nd_assemble_kernel<<<g2, 256, 0, s>>>(nF, c, per, d_asm_ + b.asm_off, d_emap_, d_fronts_);
                }
            }
          if (b.nE > 0)
            {
              double **pEE = d_ptr_ + b.ptr_off, **pEK = pEE + nb, **pKE = pEK + nb, **pKK = pKE + nb;
              int     *piv = d_piv_ + b.piv_off;
              int     *inf = d_info_ + info_base;
              if (b.fused)
                {
                  nd_small_fused_kernel<<<nb, 256, nd_fused_smem(nF), s>>>(b.nE, b.nK, d_asm_ + b.asm_off, d_emap_,
                                                                          inf, d_fronts_);
                  info_base += nb;
                  continue;
                }
              if (b.small)
                {
                  // register caps by front shape (measured per tree level on
                  // the 256 x 256 degree-2 diode)
                  const size_t sm = small_smem(b.nE, b.nK);
                  if (b.nE <= 18 && b.nK <= 72)
                    nd_small_front_capped_kernel<5><<<nb, 256, sm, s>>>(b.nE, b.nK, d_sol_ + b.sol_off, inf, d_fronts_);
                  else if (b.nE <= 18)
                    nd_small_front_capped_kernel<4><<<nb, 256, sm, s>>>(b.nE, b.nK, d_sol_ + b.sol_off, inf, d_fronts_);
                  else
                    nd_small_front_kernel<<<nb, 256, sm, s>>>(b.nE, b.nK, d_sol_ + b.sol_off, inf, d_fronts_);
                  info_base += nb;
                  continue;
                }
              if (b.big)
                {
                  int r;
                  if ((r = big_batch(b, info_base, s, err)))
                    return r;
                  info_base += nb;
                  continue;
                }
              if (b.mid)
                {
                  nd_mid_front_kernel<<<nb, NDMidTPB, nd_mid_smem(b.nE), s>>>(b.nE, b.nK, d_sol_ + b.sol_off,
                                                                             inf, d_fronts_);
                  int r;
                  if (b.nK > 0 && (r = schur_update(b, pKE, pEK, pKK, s, err)))
                    return r;
                  info_base += nb;
                  continue;
                }
              if (b.nE <= NDLuMaxE)
                nd_lu_front_kernel<<<nb, NDLuTPB, nd_lu_smem(b.nE), s>>>(b.nE, nF, d_sol_ + b.sol_off, piv, inf,
                                                                        d_fronts_);
              else if (cublasDgetrfBatched(blas_, b.nE, pEE, nF, piv, inf, nb) != CUBLAS_STATUS_SUCCESS)
                return bad(err, "cublasDgetrfBatched failed", DDHDG_SOLVER_ERROR);
              // W = U^-1 L^-1 P [F_EK | r_E]: the row permutation by a
              // coalesced in-place gather, then two triangular solves
              int *perm = d_perm_ + b.piv_off;
              nd_pivperm_kernel<<<(nb + 127) / 128, 128, 0, s>>>(nb, b.nE, piv, perm);
              {
                const dim3 g2(nb, (b.nK + 1 + NDPermCols - 1) / NDPermCols);
                nd_rowperm_kernel<<<g2, 256, b.nE * sizeof(double), s>>>(b.nE, nF, d_sol_ + b.sol_off,
                                                                         perm, d_fronts_);
              }
              int r;
              if ((r = solve_w(b, pEE, pEK, s, err)))
                return r;
              if (b.nK > 0 && (r = schur_update(b, pKE, pEK, pKK, s, err)))
                return r;
            }
          info_base += nb;
        }
      // downward pass
      for (auto it = batches_.rbegin(); it != batches_.rend(); ++it)
        {
          const auto &b = *it;
          if (b.nE == 0)
            continue;
          const int nF = b.nE + b.nK;
          int       R, S;
          nd_backsolve_shape(b.nE, b.nK, R, S);
          const dim3 g2((unsigned)b.nodes.size(), (b.nE + R - 1) / R);
          nd_backsolve_kernel<<<g2, R * S, (size_t)(b.nK + R * S) * sizeof(double), s>>>(
            nF, b.nE, R, d_sol_ + b.sol_off, d_fdofs_, d_fronts_, x);
        }
      if (cudaGetLastError() != cudaSuccess)
        return bad(err, "nested-dissection kernel launch failed", DDHDG_CUDA_ERROR);
      return DDHDG_OK;
    }

  public:
    // singular fronts (outside any graph: a host read)
    int
    check_info(cudaStream_t s, std::string &err)
    {
      std::vector<int> info(nodes_info_);
      if (cudaMemcpyAsync(info.data(), d_info_, nodes_info_ * sizeof(int), cudaMemcpyDeviceToHost, s) !=
            cudaSuccess ||
          cudaStreamSynchronize(s) != cudaSuccess)
        return bad(err, "nested-dissection solve failed", DDHDG_CUDA_ERROR);
      for (int v : info)
        if (v != 0)
          return bad(err, "global trace matrix is singular (zero pivot in a front)", DDHDG_SOLVER_ERROR);
      return DDHDG_OK;
    }

  private:

    static constexpr int NSide = 8; // side streams for the large fronts

    struct Node
    {
      int                  lo[3], hi[3];
      int                  child[2] = {-1, -1};
      int                  height   = 0;
      int64_t              cell     = -1;
      unsigned             pmask    = 0;
      int                  nE = 0, nK = 0;
      std::vector<int32_t> dofs; // [E..., K...]
      int64_t              off = 0, doff = 0, moff[2] = {0, 0};
    };
    struct Batch
    {
      int              height = 0, nE = 0, nK = 0;
      std::vector<int> nodes;
      int64_t          front_off = 0, front_end = 0, piv_off = 0, asm_off = 0, sol_off = 0, ptr_off = 0;
      bool             big     = false;
      int              maxc[2] = {0, 0}; // max child nK + 1 per extend-add pass
      bool             small   = false;  // fused one-CTA elimination
      bool             mid     = false;  // one-CTA LU + W, batched GEMM Schur update
      bool             fused   = false;  // small, assembled and eliminated in shared memory
    };

    static size_t
    small_smem(int nE, int nK)
    {
      return ((size_t)nE * nE + (size_t)nE * (nK + 1)) * sizeof(double);
    }

    // the large fronts of one batch (few, independent, each too small to
    // fill the GPU alone): LU, row permutation, triangular solves and the
    // Schur update per front, spread over the side streams
    int
    big_batch(const Batch &b, int info_base, cudaStream_t s, std::string &err)
    {
      const int nF = b.nE + b.nK;
      const int nb = (int)b.nodes.size();
      if (cudaEventRecord(ev_fork_, s) != cudaSuccess)
        return bad(err, "cudaEventRecord failed", DDHDG_CUDA_ERROR);
      const int used = std::min(nb, nside_);
      for (int k = 0; k < used; ++k)
        if (cudaStreamWaitEvent(side_[k], ev_fork_, 0) != cudaSuccess)
          return bad(err, "cudaStreamWaitEvent failed", DDHDG_CUDA_ERROR);
      const double one = 1., mone = -1.;
      for (int q = 0; q < nb; ++q)
        {
          const int    k   = q % nside_;
          cudaStream_t ss  = side_[k];
          double      *Fq  = d_fronts_ + nodes_[b.nodes[q]].off;
          int         *piv = d_piv_ + b.piv_off + (int64_t)q * b.nE;
          int         *pm  = d_perm_ + b.piv_off + (int64_t)q * b.nE;
          if (cusolverDnDgetrf(side_dn_[k], b.nE, b.nE, Fq, nF, d_work_ + (int64_t)k * work_per_,
                               piv, d_info_ + info_base + q) != CUSOLVER_STATUS_SUCCESS)
            return bad(err, "cusolverDnDgetrf failed", DDHDG_SOLVER_ERROR);
          nd_pivperm_kernel<<<1, 32, 0, ss>>>(1, b.nE, piv, pm);
          const dim3 g2(1, (b.nK + 1 + NDPermCols - 1) / NDPermCols);
          nd_rowperm_kernel<<<g2, 256, b.nE * sizeof(double), ss>>>(b.nE, nF, d_sol_ + b.sol_off + q,
                                                                    pm, d_fronts_);
          if (own_trsm_)
            continue; // W for all fronts at once, below
          double *B = Fq + (int64_t)b.nE * nF;
          if (cublasDtrsm(side_blas_[k], CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_N,
                          CUBLAS_DIAG_UNIT, b.nE, b.nK + 1, &one, Fq, nF, B, nF) != CUBLAS_STATUS_SUCCESS ||
              cublasDtrsm(side_blas_[k], CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N,
                          CUBLAS_DIAG_NON_UNIT, b.nE, b.nK + 1, &one, Fq, nF, B, nF) != CUBLAS_STATUS_SUCCESS)
            return bad(err, "cublasDtrsm failed", DDHDG_SOLVER_ERROR);
          if (own_gemm_)
            continue; // the Schur updates of all fronts at once, below
          if (b.nK > 0 &&
              cublasDgemm(side_blas_[k], CUBLAS_OP_N, CUBLAS_OP_N, b.nK, b.nK + 1, b.nE, &mone, Fq + b.nE,
                          nF, B, nF, &one, B + b.nE, nF) != CUBLAS_STATUS_SUCCESS)
            return bad(err, "cublasDgemm failed", DDHDG_SOLVER_ERROR);
        }
      for (int k = 0; k < used; ++k)
        if (cudaEventRecord(ev_join_[k], side_[k]) != cudaSuccess ||
            cudaStreamWaitEvent(s, ev_join_[k], 0) != cudaSuccess)
          return bad(err, "stream join failed", DDHDG_CUDA_ERROR);
      double **pEE = d_ptr_ + b.ptr_off, **pEK = pEE + nb, **pKE = pEK + nb, **pKK = pKE + nb;
      int      r;
      if (own_trsm_ && (r = solve_w(b, pEE, pEK, s, err)))
        return r;
      if ((own_trsm_ || own_gemm_) && b.nK > 0 && (r = schur_update(b, pKE, pEK, pKK, s, err)))
        return r;
      return DDHDG_OK;
    }

    // W = U^-1 L^-1 [F_EK | r_E] for every front of a batch (after the row
    // permutation), by the tensor-path kernels or by batched cuBLAS
    int
    solve_w(const Batch &b, double **pEE, double **pEK, cudaStream_t s, std::string &err)
    {
      const int nF = b.nE + b.nK;
      const int nb = (int)b.nodes.size();
      // each CTA of nd_trsm_kernel sweeps the whole column of blocks of its
      // 32 right-hand sides: worth it while there are enough of them (not
      // for the root's single column, nor for the largest 3D fronts)
      const int ntiles = (b.nK + 1 + NDTB - 1) / NDTB;
      if (own_trsm_ && (int64_t)ntiles * nb >= 64 && b.nE <= 1152)
        {
          const int nblk = (b.nE + NDTB - 1) / NDTB;
          nd_trinv_kernel<<<dim3(nblk, nb), 64, 0, s>>>(b.nE, nF, pEE, d_tinv_);
          nd_trsm_kernel<<<dim3((b.nK + 1 + NDTB - 1) / NDTB, nb), 128, 0, s>>>(b.nE, b.nK + 1, nF, pEE, pEK,
                                                                                 d_tinv_);
          return DDHDG_OK;
        }
      const double one_ = 1.;
      if (cublasDtrsmBatched(blas_, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_N, CUBLAS_DIAG_UNIT,
                             b.nE, b.nK + 1, &one_, pEE, nF, pEK, nF, nb) != CUBLAS_STATUS_SUCCESS ||
          cublasDtrsmBatched(blas_, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N,
                             CUBLAS_DIAG_NON_UNIT, b.nE, b.nK + 1, &one_, pEE, nF, pEK, nF,
                             nb) != CUBLAS_STATUS_SUCCESS)
        return bad(err, "cublasDtrsmBatched failed", DDHDG_SOLVER_ERROR);
      return DDHDG_OK;
    }

    // F_KK -= F_KE W for every front of a batch
    int
    schur_update(const Batch &b, double **pKE, double **pEK, double **pKK, cudaStream_t s, std::string &err)
    {
      const int nF = b.nE + b.nK;
      const int nb = (int)b.nodes.size();
      if (own_gemm_ || own_trsm_)
        {
          const int tiles = ((b.nK + NDGM - 1) / NDGM) * ((b.nK + 1 + NDGN - 1) / NDGN);
          nd_gemm_kernel<<<dim3(tiles, nb), 128, 0, s>>>(b.nK, b.nK + 1, b.nE, nF, pKE, pEK, pKK);
          return DDHDG_OK;
        }
      const double mone = -1., one = 1.;
      if (cublasDgemmBatched(blas_, CUBLAS_OP_N, CUBLAS_OP_N, b.nK, b.nK + 1, b.nE, &mone, pKE, nF, pEK, nF,
                             &one, pKK, nF, nb) != CUBLAS_STATUS_SUCCESS)
        return bad(err, "cublasDgemmBatched failed", DDHDG_SOLVER_ERROR);
      return DDHDG_OK;
    }


    static int
    bad(std::string &err, const char *msg, int code = DDHDG_BAD_ARG)
    {
      err = msg;
      return code;
    }

    int64_t
    face_at(int a, const int co[3]) const
    {
      int64_t idx = 0, stride = 1;
      for (int b = 0; b < M_.dim; ++b)
        {
          idx += co[b] * stride;
          stride *= M_.face_ext[a][b];
        }
      return M_.face_off[a] + idx;
    }

    int64_t
    face_of_cell(int64_t cell, int f) const
    {
      int       co[3];
      const int n1 = M_.dim > 1 ? M_.n[1] : 1;
      co[0]        = (int)(cell % M_.n[0]);
      co[1]        = (int)((cell / M_.n[0]) % n1);
      co[2]        = (int)(cell / ((int64_t)M_.n[0] * n1));
      co[f / 2] += f % 2;
      return face_at(f / 2, co);
    }

    // faces of axis a at face coordinate p, over the box's extent in the
    // other axes, in increasing id order
    void
    plane_faces(int a, int p, const int lo[3], const int hi[3], std::vector<int64_t> &out) const
    {
      int co[3];
      int l[3], h[3];
      for (int b = 0; b < 3; ++b)
        {
          l[b] = (b == a) ? p : lo[b];
          h[b] = (b == a) ? p + 1 : hi[b];
        }
      for (co[2] = l[2]; co[2] < h[2]; ++co[2])
        for (co[1] = l[1]; co[1] < h[1]; ++co[1])
          for (co[0] = l[0]; co[0] < h[0]; ++co[0])
            out.push_back(face_at(a, co));
    }

    void
    expand(const std::vector<int64_t> &faces, std::vector<int32_t> &dofs) const
    {
      for (int64_t f : faces)
        for (int j = 0; j < M_.nd; ++j)
          dofs.push_back((int32_t)(f * M_.nd + j));
    }

    int
    make_node(const int lo[3], const int hi[3])
    {
      const int id = (int)nodes_.size();
      nodes_.emplace_back();
      for (int b = 0; b < 3; ++b)
        {
          nodes_[id].lo[b] = lo[b];
          nodes_[id].hi[b] = hi[b];
        }
      const int ext[3] = {hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]};
      if (ext[0] * ext[1] * ext[2] == 1)
        {
          // leaf: one cell; faces on the physical boundary first
          const int     n1   = M_.dim > 1 ? M_.n[1] : 1;
          const int64_t cell = lo[0] + (int64_t)M_.n[0] * (lo[1] + (int64_t)n1 * lo[2]);
          std::vector<int64_t> E, K;
          unsigned             msk = 0;
          for (int f = 0; f < M_.F; ++f)
            {
              const int a = f / 2, p = (f % 2) ? hi[a] : lo[a];
              if (p == 0 || p == M_.n[a])
                msk |= 1u << f;
            }
          for (int f = 0; f < M_.F; ++f)
            ((msk & (1u << f)) ? E : K).push_back(cell_faces_[cell * M_.F + f]);
          auto &nd = nodes_[id];
          nd.cell  = cell;
          nd.pmask = msk;
          expand(E, nd.dofs);
          nd.nE = (int)nd.dofs.size();
          expand(K, nd.dofs);
          nd.nK     = (int)nd.dofs.size() - nd.nE;
          nd.height = 0;
          return id;
        }
      int s = 0;
      for (int b = 1; b < M_.dim; ++b)
        if (ext[b] > ext[s])
          s = b;
      const int mid   = lo[s] + ext[s] / 2;
      int       hl[3] = {hi[0], hi[1], hi[2]}, lh[3] = {lo[0], lo[1], lo[2]};
      hl[s]           = mid;
      lh[s]           = mid;
      const int c0    = make_node(lo, hl);
      const int c1    = make_node(lh, hi);
      std::vector<int64_t> E, K;
      plane_faces(s, mid, lo, hi, E);
      for (int a = 0; a < M_.dim; ++a)
        {
          if (lo[a] > 0)
            plane_faces(a, lo[a], lo, hi, K);
          if (hi[a] < M_.n[a])
            plane_faces(a, hi[a], lo, hi, K);
        }
      std::sort(K.begin(), K.end());
      auto &nd    = nodes_[id]; // after the recursion: nodes_ may have grown
      nd.child[0] = c0;
      nd.child[1] = c1;
      expand(E, nd.dofs);
      nd.nE = (int)nd.dofs.size();
      expand(K, nd.dofs);
      nd.nK     = (int)nd.dofs.size() - nd.nE;
      nd.height = 1 + std::max(nodes_[c0].height, nodes_[c1].height);
      return id;
    }

    template <typename T>
    int
    dmalloc(T *&p, size_t bytes, std::string &err)
    {
      if (cudaMalloc(reinterpret_cast<void **>(&p), std::max<size_t>(bytes, 16)) != cudaSuccess)
        {
          cudaGetLastError();
          p   = nullptr;
          err = "cudaMalloc of " + std::to_string(bytes) + " bytes for the trace solver failed";
          return DDHDG_OOM;
        }
      allocs_.push_back(p);
      return DDHDG_OK;
    }

    template <typename T>
    int
    upload(T *&p, const std::vector<T> &v, std::string &err)
    {
      int r = dmalloc(p, v.size() * sizeof(T), err);
      if (r)
        return r;
      if (!v.empty() && cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess)
        return bad(err, "upload failed", DDHDG_CUDA_ERROR);
      return DDHDG_OK;
    }

    void
    release()
    {
      for (void *p : allocs_)
        cudaFree(p);
      allocs_.clear();
      if (blas_)
        cublasDestroy(blas_);
      blas_  = nullptr;
      for (int k = 0; k < NSide; ++k)
        {
          if (side_blas_[k])
            cublasDestroy(side_blas_[k]);
          if (side_dn_[k])
            cusolverDnDestroy(side_dn_[k]);
          if (ev_join_[k])
            cudaEventDestroy(ev_join_[k]);
          if (side_[k])
            cudaStreamDestroy(side_[k]);
          side_blas_[k] = nullptr;
          side_dn_[k]   = nullptr;
          ev_join_[k]   = nullptr;
          side_[k]      = nullptr;
        }
      if (ev_fork_)
        cudaEventDestroy(ev_fork_);
      ev_fork_ = nullptr;
      if (exec_)
        cudaGraphExecDestroy(exec_);
      exec_ = nullptr;
      if (cap_)
        cudaStreamDestroy(cap_);
      cap_       = nullptr;
      key_       = Key{};
      graphs_ok_ = true;
      built_ = false;
    }

    // a cached plan: the members that plan_uncached fills
    struct PlanState
    {
      Mesh                 M;
      std::vector<Node>    nodes;
      std::vector<Batch>   batches;
      std::vector<int64_t> cell_faces;
      int                  root = -1, max_nK = 0;
      int64_t              front_total = 0, piv_total = 0;
      std::vector<int32_t> fdofs, emap;
      std::vector<int64_t> leaf_off, ptr;
      std::vector<uint8_t> pmask;
      std::vector<NDAsm>   asm_;
      std::vector<NDSol>   sol;
      size_t
      bytes() const
      {
        size_t b = cell_faces.size() * 8 + fdofs.size() * 4 + emap.size() * 4 + leaf_off.size() * 8 +
                   ptr.size() * 8 + pmask.size() + asm_.size() * sizeof(NDAsm) + sol.size() * sizeof(NDSol);
        for (const auto &n : nodes)
          b += sizeof(Node) + n.dofs.size() * 4;
        for (const auto &bt : batches)
          b += sizeof(Batch) + bt.nodes.size() * 4;
        return b;
      }
    };
    void
    save_plan(PlanState &e) const
    {
      e.M           = M_;
      e.nodes       = nodes_;
      e.batches     = batches_;
      e.cell_faces  = cell_faces_;
      e.root        = root_;
      e.max_nK      = max_nK_;
      e.front_total = front_total_;
      e.piv_total   = piv_total_;
      e.fdofs       = fdofs_h_;
      e.emap        = emap_h_;
      e.leaf_off    = leaf_off_h_;
      e.ptr         = ptr_h_;
      e.pmask       = pmask_h_;
      e.asm_        = asm_h_;
      e.sol         = sol_h_;
    }
    void
    load_plan(const PlanState &e)
    {
      M_           = e.M;
      nodes_       = e.nodes;
      batches_     = e.batches;
      cell_faces_  = e.cell_faces;
      root_        = e.root;
      max_nK_      = e.max_nK;
      front_total_ = e.front_total;
      piv_total_   = e.piv_total;
      fdofs_h_     = e.fdofs;
      emap_h_      = e.emap;
      leaf_off_h_  = e.leaf_off;
      ptr_h_       = e.ptr;
      pmask_h_     = e.pmask;
      asm_h_       = e.asm_;
      sol_h_       = e.sol;
    }

    Mesh                 M_;
    std::vector<Node>    nodes_;
    std::vector<Batch>   batches_;
    std::vector<int64_t> cell_faces_;
    int                  root_ = -1, nodes_info_ = 0, max_nK_ = 0;
    int64_t              front_total_ = 0, piv_total_ = 0;
    bool                 built_       = false;
    // host copies of the plan (uploaded by build)
    std::vector<int32_t> fdofs_h_, emap_h_;
    std::vector<int64_t> leaf_off_h_, ptr_h_;
    std::vector<uint8_t> pmask_h_;
    std::vector<NDAsm>   asm_h_;
    std::vector<NDSol>   sol_h_;
    // device
    std::vector<void *> allocs_;
    double             *d_fronts_ = nullptr, *d_dscale_ = nullptr, *d_work_ = nullptr;
    double             *d_tinv_   = nullptr; // inverted diagonal blocks of the triangular solves
    bool                own_trsm_ = false;   // tensor-path triangular solves for W
    bool                own_gemm_ = false;   // tensor-path Schur updates
    double            **d_ptr_    = nullptr;
    int                *d_piv_ = nullptr, *d_perm_ = nullptr, *d_info_ = nullptr;
    int32_t            *d_fdofs_ = nullptr, *d_emap_ = nullptr;
    int64_t            *d_leaf_off_ = nullptr, *d_cell_faces_ = nullptr;
    uint8_t            *d_pmask_ = nullptr;
    NDAsm              *d_asm_   = nullptr;
    NDSol              *d_sol_   = nullptr;
    unsigned long long *d_dmax_  = nullptr;
    cublasHandle_t      blas_    = nullptr;
    int                 nside_            = 0; // side streams created (side_count())
    cudaStream_t        side_[NSide]      = {};
    cublasHandle_t      side_blas_[NSide] = {};
    cusolverDnHandle_t  side_dn_[NSide]   = {};
    cudaEvent_t         ev_join_[NSide]   = {};
    cudaEvent_t         ev_fork_          = nullptr;
    int64_t             work_per_         = 1;
    cudaStream_t        cap_              = nullptr; // stream the graph is captured on
    cudaGraphExec_t     exec_             = nullptr;
    Key                 key_{};
    bool                graphs_ok_ = true;  // capture works in this build
    bool                use_graphs_ = true; // the caller wants graphs
  };
} // namespace ddhdg
