// Batched condensation and reconstruction: many devices (diodes) of
// different mesh sizes and polynomial degrees in one persistent launch per
// Newton step.
//
// The reference assembles one device at a time, its per-cell worker run over
// the cells by WorkStream (include/assembling_methods.template.h:67-88).
// Here a work list of tiles (device, range of its cells) is consumed by one
// grid of CTAs of BatchTPB threads: every CTA takes the next tile from a
// counter, loads that device's launch parameters into shared memory and runs
// the per-degree body on the tile's cells (the unit-cell constant tables of
// every degree travel in the constant bank): two warps on two cells at a time
// for the warp-per-cell degrees (condense3_cells, FP64 or with the FP32
// Jacobian of a mixed-precision device), the whole CTA on one cell at a time
// otherwise (condense2_cells).  Tiles are ordered heaviest first; their sizes
// per degree and the CTAs per SM come from the host's autotuner.  Every
// device's results are bitwise those of its own ddhdg_assemble_condense (same
// tables, same parameters, same arithmetic).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>
#include <type_traits>

#include "hdg_condense.cuh"
#include "hdg_condense3.cuh"
#include "hdg_kernels.cuh"

namespace ddhdg
{
  constexpr int BatchTPB  = 64;          // 2 warps: two cells at a time, or one CTA-per-cell cell
  constexpr int BatchWarp = BatchTPB / 32;
  constexpr int BatchRTPB = 256;         // reconstruction: 8 warps

  struct BatchJob
  {
    KParams       P;      // the device's parameters: state, outputs, tables, Y cache
    const double *dtrace; // reconstruction: trace update [nfaces][3][nf]
    double       *dcell;  // reconstruction: cell update [ncells][Nc_all]
    int           k;
    int           mixed;  // 1: FP32 Jacobian (condense3_cells<..., float>)
  };

  struct BatchTile
  {
    int32_t job;
    int32_t pad;
    int64_t begin, end;
  };

  // the CTA copies a job's parameters into shared memory
  __device__ __forceinline__ void
  batch_load_params(KParams &dst, const KParams &src)
  {
    static_assert(sizeof(KParams) % 8 == 0, "KParams is copied as 8-byte words");
    const unsigned long long *s = reinterpret_cast<const unsigned long long *>(&src);
    unsigned long long       *d = reinterpret_cast<unsigned long long *>(&dst);
    for (int i = threadIdx.x; i < (int)(sizeof(KParams) / 8); i += blockDim.x)
      d[i] = s[i];
  }

  // (dim, degree) pairs with a condensation kernel
  template <int DIM, int K>
  constexpr bool batch_has = (DIM <= 2 && K >= 1 && K <= 3) || (DIM == 3 && (K == 1 || K == 2));
  template <int DIM, int K>
  constexpr bool batch_warp = batch_has<DIM, K> && 3 * Dims<DIM, K>::nb <= 32;

  // The unit-cell constant tables of the warp-per-cell degrees of one
  // dimension: the same for every device of that degree (the mesh size
  // enters through KParams::ih), so one copy travels in the constant bank
  struct NoTab
  {
  };
  template <int DIM>
  struct BatchTabs
  {
    std::conditional_t<batch_warp<DIM, 1>, CTab<DIM, 1>, NoTab> t1;
    std::conditional_t<batch_warp<DIM, 2>, CTab<DIM, 2>, NoTab> t2;
    std::conditional_t<batch_warp<DIM, 3>, CTab<DIM, 3>, NoTab> t3;
  };
  template <int K, int DIM>
  __host__ __device__ __forceinline__ const auto &
  batch_tab(const BatchTabs<DIM> &C)
  {
    if constexpr (K == 1)
      return C.t1;
    else if constexpr (K == 2)
      return C.t2;
    else
      return C.t3;
  }

  // JT: the Jacobian type of the warp-per-cell body (the CTA-per-cell
  // degrees are FP64 only)
  template <int DIM, int K, typename JT>
  __device__ __forceinline__ void
  batch_condense_tile(const KParams &P, const BatchTabs<DIM> &C, const BatchTile &t, double *smem,
                      int (*piv)[32])
  {
    if constexpr (!batch_has<DIM, K>)
      return;
    else if constexpr (batch_warp<DIM, K>)
      {
        const int    warp = threadIdx.x >> 5;
        const Ws3Off wo   = ws3_layout(DIM, Dims<DIM, K>::nb, Dims<DIM, K>::nf, P.ncomp, P.ncol, (int)sizeof(JT));
        // the device's face-flux table of the tt epilogue, after the warps'
        // workspaces (as the single-device kernel stages it)
        constexpr int NR  = CTab<DIM, K>::Fq * CTab<DIM, K>::Ft;
        double       *rqr = smem + BatchWarp * wo.total;
        for (int i = threadIdx.x; i < NR; i += BatchTPB)
          rqr[i] = P.tables[P.to.RQr + i];
        __syncthreads();
        condense3_cells<DIM, K, JT>(P, batch_tab<K>(C), smem + warp * wo.total, piv[warp], t.begin + warp,
                                    t.end, BatchWarp, rqr);
      }
    else if constexpr (sizeof(JT) == 8)
      condense2_cells<DIM, K, BatchTPB>(P, smem, blockIdx.x, t.begin, t.end, 1);
  }

  // The precisions a batch holds: FP64 devices only, mixed-precision
  // warp-per-cell devices only, or both.  Each class is its own
  // instantiation, so that a batch carries only the bodies it runs: the
  // mixed-only kernel is built for eight CTAs of two warps per SM (128
  // registers), the occupancy of the single-device mixed kernel; the others
  // for four (the FP64 bodies take 255 registers, and the mixed bodies
  // beside them add spills).  Small CTAs keep several CTA-per-cell cells
  // on an SM, so that their serial LU panels overlap.
  enum BatchPrec : int
  {
    BatchFP64  = 0,
    BatchMixed = 1,
    BatchBoth  = 2
  };

  // counter: tiles handed out so far (zero at launch)
  template <int DIM, int PREC>
  __global__ void __launch_bounds__(BatchTPB, PREC == BatchMixed ? 8 : 4)
  batch_condense_kernel(const BatchJob *__restrict__ jobs, const BatchTile *__restrict__ tiles,
                        int ntiles, int *counter, const __grid_constant__ BatchTabs<DIM> C)
  {
    extern __shared__ __align__(16) double smem[];
    __shared__ int                   piv[BatchWarp][32];
    __shared__ __align__(16) KParams Ps;
    __shared__ int                   s_tile, s_k;
    for (;;)
      {
        __syncthreads(); // the previous tile is done with Ps and the workspace
        if (threadIdx.x == 0)
          s_tile = atomicAdd(counter, 1);
        __syncthreads();
        const int ti = s_tile;
        if (ti >= ntiles)
          break;
        const BatchTile t = tiles[ti];
        batch_load_params(Ps, jobs[t.job].P);
        if (threadIdx.x == 0)
          s_k = jobs[t.job].k + (jobs[t.job].mixed ? 4 : 0);
        __syncthreads();
        const int sk = s_k;
        if constexpr (PREC != BatchMixed)
          {
            if (sk == 1)
              batch_condense_tile<DIM, 1, double>(Ps, C, t, smem, piv);
            else if (sk == 2)
              batch_condense_tile<DIM, 2, double>(Ps, C, t, smem, piv);
            else if (sk == 3)
              batch_condense_tile<DIM, 3, double>(Ps, C, t, smem, piv);
          }
        if constexpr (PREC != BatchFP64)
          {
            if (sk == 5)
              batch_condense_tile<DIM, 1, float>(Ps, C, t, smem, piv);
            else if (sk == 6)
              batch_condense_tile<DIM, 2, float>(Ps, C, t, smem, piv);
            else if (sk == 7)
              batch_condense_tile<DIM, 3, float>(Ps, C, t, smem, piv);
          }
      }
  }

  template <int DIM>
  __global__ void __launch_bounds__(BatchRTPB, 4)
  batch_reconstruct_kernel(const BatchJob *__restrict__ jobs, const BatchTile *__restrict__ tiles,
                           int ntiles, int *counter)
  {
    extern __shared__ __align__(16) double smem[];
    __shared__ __align__(16) KParams Ps;
    __shared__ int                   s_tile, s_k;
    __shared__ const double         *s_dt;
    __shared__ double               *s_dc;
    for (;;)
      {
        __syncthreads(); // the previous tile is done with Ps and the staged operators
        if (threadIdx.x == 0)
          s_tile = atomicAdd(counter, 1);
        __syncthreads();
        const int ti = s_tile;
        if (ti >= ntiles)
          break;
        const BatchTile t = tiles[ti];
        batch_load_params(Ps, jobs[t.job].P);
        if (threadIdx.x == 0)
          {
            s_k  = jobs[t.job].k;
            s_dt = jobs[t.job].dtrace;
            s_dc = jobs[t.job].dcell;
          }
        __syncthreads();
        const int64_t nw = blockDim.x >> 5;
        switch (s_k)
          {
            case 1: reconstruct_cells<DIM, 1>(Ps, s_dt, s_dc, smem, t.begin, 1, t.end, nw); break;
            case 2: reconstruct_cells<DIM, 2>(Ps, s_dt, s_dc, smem, t.begin, 1, t.end, nw); break;
            case 3:
              if constexpr (batch_has<DIM, 3>)
                reconstruct_cells<DIM, 3>(Ps, s_dt, s_dc, smem, t.begin, 1, t.end, nw);
              break;
            default: break;
          }
      }
  }
} // namespace ddhdg
