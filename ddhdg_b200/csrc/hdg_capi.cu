// C ABI of the B200 HDG hot path: context set-up (NPSolver construction and
// setup_overall_system, src/np_solver.cpp:553-655), the per-cell
// condensation and reconstruction launches, the global trace assembly
// (copy_local_to_global, src/np_solver.cpp:1293-1322), the global trace
// solve (solve_linear_problem, src/np_solver.cpp:1326-1354) and the Newton
// loop (private_run, src/np_solver.cpp:1452-1561).
#include <cuda_runtime.h>
#include <cusolverSp.h>
#include <cusparse.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <memory>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/ddhdg_b200.h"
#include "hdg_batch.cuh"
#include "hdg_condense.cuh"
#include "hdg_condense3.cuh"
#include "hdg_kernels.cuh"
#include "hdg_ndsolve.cuh"
#include "hdg_plain.cuh"
#include "hdg_tables.h"

using namespace ddhdg;

namespace
{
  thread_local std::string g_last_error;

  int
  fail(int code, const std::string &msg)
  {
    g_last_error = msg;
    return code;
  }

#define CK(call)                                                              \
  do                                                                          \
    {                                                                         \
      cudaError_t e_ = (call);                                                \
      if (e_ != cudaSuccess)                                                  \
        return fail(DDHDG_CUDA_ERROR, std::string(#call) + ": " +             \
                                        cudaGetErrorString(e_));              \
    }                                                                         \
  while (0)

  template <typename T>
  struct DevBuf
  {
    T     *p = nullptr;
    size_t n = 0;
    int
    alloc(size_t count)
    {
      if (count <= n && p)
        return DDHDG_OK;
      if (p)
        cudaFree(p);
      p = nullptr;
      n = 0;
      if (count == 0)
        return DDHDG_OK;
      if (cudaMalloc(&p, count * sizeof(T)) != cudaSuccess)
        {
          cudaGetLastError();
          return fail(DDHDG_OOM, "cudaMalloc of " + std::to_string(count * sizeof(T)) + " bytes failed");
        }
      n = count;
      return DDHDG_OK;
    }
    int
    upload(const T *h, size_t count)
    {
      int r = alloc(count);
      if (r)
        return r;
      if (count && cudaMemcpy(p, h, count * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess)
        return fail(DDHDG_CUDA_ERROR, "upload failed");
      return DDHDG_OK;
    }
    void
    release()
    {
      if (p)
        cudaFree(p);
      p = nullptr;
      n = 0;
    }
    ~DevBuf() { release(); }
  };

  // per mode (0: regular run, 1: thermodynamic equilibrium = V only)
  struct Mode
  {
    int                   comps[3] = {0, 1, 2};
    int                   ncomp    = 0;
    int                   Nt       = 0;
    int                   ncol     = 0;
    int                   ycols    = 0;
    int64_t               ndofs    = 0;
    int64_t               nnz      = 0;
    DevBuf<int32_t>       rowptr, colind;
    DevBuf<uint8_t>       slots; // [ncells][F][F]
    DevBuf<double>        ycache, tt, rhs, dval, csr, grhs, x, dtrace, dcell;
    DevBuf<double>        rscratch; // per-CTA R blocks of the condense kernel, if needed
    std::unique_ptr<NDSolver> nd;   // nested-dissection trace solver (built on first use)
    DevBuf<int32_t>       dflag;
    std::vector<int32_t>  perm; // nested-dissection order of the trace dofs
    DevBuf<int32_t>       d_perm, d_iperm, prow, pcol;
    DevBuf<int32_t>       pmap; // permuted position of each CSR entry
    DevBuf<double>        pval, pb, px;
    bool                  built = false;
  };
} // namespace

struct ddhdg_ctx
{
  ddhdg_problem_desc desc{};
  int                dim = 0, k = 0, nb = 0, nf = 0, nqc = 0, nqf = 0, F = 0;
  int64_t            ncells = 0, nfaces = 0;
  int64_t            face_off[3]    = {0, 0, 0};
  int                face_ext[3][3] = {{1, 1, 1}, {1, 1, 1}, {1, 1, 1}};
  int                enabled[3]     = {1, 1, 1};
  Tables             T;
  Tables             Tu; // the same tables on the unit cell (constant-bank copies)
  TabOff             to{};
  DevBuf<double>     tables, doping, rec_a, rec_b, rec_c, tau_table, bc_val;
  DevBuf<int32_t>    bc;
  DevBuf<int>        status;
  Mode               mode[2];
  int                sm_count = 148;
  cusolverSpHandle_t sp       = nullptr;
  cusparseMatDescr_t descr    = nullptr;
  // face -> adjacent cells
  std::vector<int64_t> face_cells; // [nfaces][2] (-1 when absent)
  bool               solver_graphs = true; // CUDA-graph capture of the trace solve
  double             t_condense = 0., t_solve = 0., t_recon = 0.;
  int                t_steps    = 0;
  DevBuf<double>     norm_buf;
  DevBuf<int64_t>    d_face_cells, d_face_local;
  // the plain (full local system) path: per-CTA workspace and tc slices
  DevBuf<double>     plain_ws, plain_tc;
  // host-buffer calls: device copies of the state and of the reconstruction
  // input and output, a copy stream per direction, events per chunk
  struct HostIO
  {
    static constexpr int NChunk = 4;
    DevBuf<double>       cell, trace, dtrace, dcell;
    cudaStream_t         h2d = nullptr, d2h = nullptr;
    cudaEvent_t          ev_trace = nullptr, ev_out = nullptr;
    // recorded after the last kernel that reads the device state copies /
    // the trace-update copy: the next upload into them waits for it only
    cudaEvent_t          ev_cell_free = nullptr, ev_dtrace_free = nullptr;
    cudaEvent_t          ev_chunk[NChunk] = {}, ev_rec[NChunk] = {};
    bool                 ready = false, have_state = false;
    ~HostIO()
    {
      for (cudaEvent_t e : {ev_trace, ev_out, ev_cell_free, ev_dtrace_free})
        if (e)
          cudaEventDestroy(e);
      for (int k = 0; k < NChunk; ++k)
        {
          if (ev_chunk[k])
            cudaEventDestroy(ev_chunk[k]);
          if (ev_rec[k])
            cudaEventDestroy(ev_rec[k]);
        }
      if (h2d)
        cudaStreamDestroy(h2d);
      if (d2h)
        cudaStreamDestroy(d2h);
    }
  } hio;
};

namespace
{
  int
  ncol_for(const ddhdg_ctx *c, const Mode &m)
  {
    return (c->desc.flux == DDHDG_FLUX_USE_CELL) ? 1 + m.Nt : 1 + 2 * m.Nt;
  }

  void
  set_mode_comps(ddhdg_ctx *c, int thermo)
  {
    Mode &m = c->mode[thermo];
    m.ncomp = 0;
    if (thermo)
      m.comps[m.ncomp++] = 0;
    else
      for (int b = 0; b < 3; ++b)
        if (c->enabled[b])
          m.comps[m.ncomp++] = b;
    m.Nt    = c->F * m.ncomp * c->nf;
    m.ncol  = ncol_for(c, m);
    m.ycols = 1 + m.Nt;
    m.ndofs = c->nfaces * m.ncomp * c->nf;
  }

  int64_t
  face_of_cell(const ddhdg_ctx *c, int64_t cell, int f)
  {
    int ci[3];
    ci[0] = (int)(cell % c->desc.n[0]);
    ci[1] = (int)((cell / c->desc.n[0]) % (c->dim > 1 ? c->desc.n[1] : 1));
    ci[2] = (int)(cell / ((int64_t)c->desc.n[0] * (c->dim > 1 ? c->desc.n[1] : 1)));
    const int a = f / 2;
    ci[a] += f % 2;
    int64_t idx = 0, stride = 1;
    for (int b = 0; b < c->dim; ++b)
      {
        idx += ci[b] * stride;
        stride *= c->face_ext[a][b];
      }
    return c->face_off[a] + idx;
  }

  // Nested-dissection order of the faces of the structured mesh: recursive
  // bisection of the cell box along its longest axis; the faces of the
  // separating plane are numbered after both halves.
  void
  nd_order(const ddhdg_ctx *c, std::vector<int64_t> &order)
  {
    std::vector<char> used(c->nfaces, 0);
    order.clear();
    order.reserve(c->nfaces);
    struct Box
    {
      int lo[3], hi[3];
    };
    // faces of a box: all faces of its cells not yet numbered
    std::function<void(Box)> rec = [&](Box b) {
      int ext[3], ax = 0, best = 0;
      int64_t ncell = 1;
      for (int a = 0; a < 3; ++a)
        {
          ext[a] = b.hi[a] - b.lo[a];
          ncell *= ext[a];
          if (a < c->dim && ext[a] > best)
            {
              best = ext[a];
              ax   = a;
            }
        }
      if (ncell <= 4 || best <= 1)
        {
          for (int z = b.lo[2]; z < b.hi[2]; ++z)
            for (int y = b.lo[1]; y < b.hi[1]; ++y)
              for (int x = b.lo[0]; x < b.hi[0]; ++x)
                {
                  const int64_t cell =
                    x + (int64_t)c->desc.n[0] * (y + (int64_t)(c->dim > 1 ? c->desc.n[1] : 1) * z);
                  for (int f = 0; f < c->F; ++f)
                    {
                      const int64_t Fi = face_of_cell(c, cell, f);
                      if (!used[Fi])
                        {
                          used[Fi] = 1;
                          order.push_back(Fi);
                        }
                    }
                }
          return;
        }
      const int mid = b.lo[ax] + ext[ax] / 2;
      // separator: faces with normal ax at position mid inside the box
      std::vector<int64_t> sep;
      int                  lo[3] = {b.lo[0], b.lo[1], b.lo[2]};
      int                  hi[3] = {b.hi[0], b.hi[1], b.hi[2]};
      lo[ax] = mid;
      hi[ax] = mid + 1;
      for (int z = lo[2]; z < hi[2]; ++z)
        for (int y = lo[1]; y < hi[1]; ++y)
          for (int x = lo[0]; x < hi[0]; ++x)
            {
              const int64_t cell =
                x + (int64_t)c->desc.n[0] * (y + (int64_t)(c->dim > 1 ? c->desc.n[1] : 1) * z);
              const int64_t Fi = face_of_cell(c, cell, 2 * ax);
              if (!used[Fi])
                {
                  used[Fi] = 1;
                  sep.push_back(Fi);
                }
            }
      Box b1 = b, b2 = b;
      b1.hi[ax] = mid;
      b2.lo[ax] = mid;
      rec(b1);
      rec(b2);
      for (auto f : sep)
        order.push_back(f);
    };
    Box all;
    for (int a = 0; a < 3; ++a)
      {
        all.lo[a] = 0;
        all.hi[a] = (a < c->dim) ? c->desc.n[a] : 1;
      }
    rec(all);
  }

  // Global trace sparsity (DoFTools::make_sparsity_pattern on the
  // restricted trace dofs, src/np_solver.cpp:643-651) and the scatter slots.
  int
  build_mode(ddhdg_ctx *c, int thermo)
  {
    Mode &m = c->mode[thermo];
    set_mode_comps(c, thermo);
    m.nd.reset();
    const int     F = c->F, nf = c->nf, nc = m.ncomp;
    const int64_t nfaces = c->nfaces;
    // neighbour faces of every face
    std::vector<std::vector<int64_t>> nbr(nfaces);
    for (int64_t f = 0; f < nfaces; ++f)
      for (int s = 0; s < 2; ++s)
        {
          const int64_t cell = c->face_cells[f * 2 + s];
          if (cell < 0)
            continue;
          for (int g = 0; g < F; ++g)
            nbr[f].push_back(face_of_cell(c, cell, g));
        }
    for (auto &v : nbr)
      {
        std::sort(v.begin(), v.end());
        v.erase(std::unique(v.begin(), v.end()), v.end());
      }
    const int64_t        ndofs = nfaces * nc * nf;
    std::vector<int32_t> rowptr(ndofs + 1, 0);
    int64_t              nnz = 0;
    for (int64_t f = 0; f < nfaces; ++f)
      for (int r = 0; r < nc * nf; ++r)
        {
          rowptr[f * nc * nf + r] = (int32_t)nnz;
          nnz += (int64_t)nbr[f].size() * nc * nf;
        }
    rowptr[ndofs] = (int32_t)nnz;
    if (nnz > INT32_MAX)
      return fail(DDHDG_BAD_ARG, "global trace matrix too large for 32-bit CSR");
    std::vector<int32_t> colind(nnz);
    for (int64_t f = 0; f < nfaces; ++f)
      for (int r = 0; r < nc * nf; ++r)
        {
          int64_t p = rowptr[f * nc * nf + r];
          for (auto g : nbr[f])
            for (int cc = 0; cc < nc * nf; ++cc)
              colind[p++] = (int32_t)(g * nc * nf + cc);
        }
    std::vector<uint8_t> slots(c->ncells * F * F);
    for (int64_t cell = 0; cell < c->ncells; ++cell)
      for (int fi = 0; fi < F; ++fi)
        {
          const int64_t Fi = face_of_cell(c, cell, fi);
          for (int fj = 0; fj < F; ++fj)
            {
              const int64_t Fj = face_of_cell(c, cell, fj);
              const auto    it = std::lower_bound(nbr[Fi].begin(), nbr[Fi].end(), Fj);
              slots[(cell * F + fi) * F + fj] = (uint8_t)(it - nbr[Fi].begin());
            }
        }
    int r;
    if ((r = m.rowptr.upload(rowptr.data(), rowptr.size())))
      return r;
    if ((r = m.colind.upload(colind.data(), colind.size())))
      return r;
    if ((r = m.slots.upload(slots.data(), slots.size())))
      return r;
    m.nnz = nnz;
    // nested-dissection permutation of the dofs for the sparse QR solve
    std::vector<int64_t> forder;
    nd_order(c, forder);
    std::vector<int32_t> perm(ndofs), iperm(ndofs);
    int64_t              q = 0;
    for (auto f : forder)
      for (int cc = 0; cc < nc * nf; ++cc)
        perm[q++] = (int32_t)(f * nc * nf + cc);
    for (int64_t i = 0; i < ndofs; ++i)
      iperm[perm[i]] = (int32_t)i;
    // permuted matrix B = A(perm, perm): rows in new order, columns renumbered
    std::vector<int32_t> prow(ndofs + 1, 0), pcol(nnz), pmap(nnz);
    int64_t              pp = 0;
    for (int64_t i = 0; i < ndofs; ++i)
      {
        prow[i]            = (int32_t)pp;
        const int64_t  old = perm[i];
        std::vector<std::pair<int32_t, int32_t>> ent;
        for (int64_t e = rowptr[old]; e < rowptr[old + 1]; ++e)
          ent.push_back({iperm[colind[e]], (int32_t)e});
        std::sort(ent.begin(), ent.end());
        for (auto &pr : ent)
          {
            pcol[pp] = pr.first;
            pmap[pp] = pr.second;
            ++pp;
          }
      }
    prow[ndofs] = (int32_t)pp;
    if ((r = m.d_perm.upload(perm.data(), perm.size())))
      return r;
    if ((r = m.d_iperm.upload(iperm.data(), iperm.size())))
      return r;
    if ((r = m.prow.upload(prow.data(), prow.size())))
      return r;
    if ((r = m.pcol.upload(pcol.data(), pcol.size())))
      return r;
    if ((r = m.pmap.upload(pmap.data(), pmap.size())))
      return r;
    m.built = true;
    return DDHDG_OK;
  }

  int
  ensure_buffers(ddhdg_ctx *c, int thermo)
  {
    Mode &m = c->mode[thermo];
    int   r;
    if (!m.built && (r = build_mode(c, thermo)))
      return r;
    const int64_t nc = c->ncells;
    const int     Ns = m.ncomp * c->nb;
    if ((r = m.ycache.alloc(nc * Ns * m.ycols)))
      return r;
    if ((r = m.tt.alloc(nc * m.Nt * m.Nt)))
      return r;
    if ((r = m.rhs.alloc(nc * m.Nt)))
      return r;
    if ((r = m.dval.alloc(nc * m.Nt)))
      return r;
    if ((r = m.dflag.alloc(nc * m.Nt)))
      return r;
    return DDHDG_OK;
  }

  KParams
  make_params(ddhdg_ctx *c, int thermo)
  {
    Mode     &m = c->mode[thermo];
    KParams   P{};
    const auto &d = c->desc;
    for (int a = 0; a < 3; ++a)
      {
        P.n[a]        = (a < c->dim) ? d.n[a] : 1;
        P.face_off[a] = c->face_off[a];
        for (int b = 0; b < 3; ++b)
          P.face_ext[a][b] = c->face_ext[a][b];
      }
    P.ncells      = c->ncells;
    for (int a = 0; a < 3; ++a)
      P.ih[a] = (a < c->dim) ? 1. / d.h[a] : 1.;
    P.tables      = c->tables.p;
    P.to          = c->to;
    P.eps         = d.eps;
    P.mun         = d.mu_n;
    P.mup         = d.mu_p;
    P.U_T         = (KB_ * d.temperature / Q_) / d.thermal_voltage_rescale;
    P.T           = d.temperature;
    P.V_rescale   = d.V_rescale;
    P.n_rescale   = d.n_rescale;
    P.rec_rescale = d.rec_rescale;
    P.nc          = d.nc;
    P.nv          = d.nv;
    P.ec          = d.ec_eV * EV_;
    P.ev          = d.ev_eV * EV_;
    P.rec_type    = d.rec_type;
    P.srh_ni      = d.srh_ni;
    P.srh_tau_n   = d.srh_tau_n;
    P.srh_tau_p   = d.srh_tau_p;
    P.rec_a       = c->rec_a.p;
    P.rec_b       = c->rec_b.p;
    P.rec_c       = c->rec_c.p;
    P.doping      = c->doping.p;
    P.tau_table   = c->tau_table.p;
    for (int b = 0; b < 3; ++b)
      P.tau[b] = d.tau[b];
    P.face_bc     = c->bc.p;
    P.face_bc_val = c->bc_val.p;
    for (int b = 0; b < 3; ++b)
      P.comps[b] = m.comps[b];
    P.ncomp         = m.ncomp;
    P.flux          = d.flux;
    P.phi_linearize = d.phi_linearize;
    P.thermo        = thermo;
    P.jfix          = d.jacobian_fix;
    P.ncol          = m.ncol;
    P.ycols         = m.ycols;
    P.status        = c->status.p;
    return P;
  }

  using ReconstructFn = void (*)(KParams, const double *, double *);

  // one condense kernel of a (dim, degree): its address (attributes,
  // occupancy) and a launcher that builds its parameters
  struct CondenseKernel
  {
    const void *fn = nullptr;
    void (*launch)(const Tables &, const KParams &, int, int, size_t, cudaStream_t) = nullptr;
  };

  template <int D, int K>
  void
  fill_ctab(const Tables &T, CTab<D, K> &C)
  {
    auto put = [](double *dst, size_t n, const std::vector<double> &src) {
      std::memcpy(dst, src.data(), std::min(n, src.size()) * sizeof(double));
    };
    put(C.phi_c, sizeof(C.phi_c) / sizeof(double), T.phi_c);
    put(C.RTk, sizeof(C.RTk) / sizeof(double), T.RTk);
    put(C.phi_f, sizeof(C.phi_f) / sizeof(double), T.phi_f);
    put(C.RTr, sizeof(C.RTr) / sizeof(double), T.RTr);
    put(C.RQk, sizeof(C.RQk) / sizeof(double), T.RQk);
    put(C.RQr, sizeof(C.RQr) / sizeof(double), T.RQr);
    put(C.xi, sizeof(C.xi) / sizeof(double), T.xi);
  }

  template <int D, int K, typename JT>
  void
  launch_condense(const Tables &T, const KParams &P, int grid, int threads, size_t smem,
                  cudaStream_t s)
  {
    if constexpr (3 * Dims<D, K>::nb <= 32)
      {
        CTab<D, K> C;
        fill_ctab(T, C);
        condense3_kernel<D, K, JT><<<grid, threads, smem, s>>>(P, C);
      }
    else
      condense2_kernel<D, K><<<grid, threads, smem, s>>>(P);
  }

  // mixed: the FP32-Jacobian variant of the warp-per-cell kernel; false when
  // the (dim, degree) has none (the caller rejects mixed precision there)
  template <int D, int K>
  bool
  pick(CondenseKernel &cf, ReconstructFn &rf, bool mixed)
  {
    // warp-per-cell register kernel when one lane can own one row of the
    // scalar system, CTA-per-cell shared-memory kernel otherwise
    rf = reconstruct_kernel<D, K>;
    if constexpr (3 * Dims<D, K>::nb <= 32)
      {
        if (mixed)
          {
            cf.fn     = reinterpret_cast<const void *>(condense3_kernel<D, K, float>);
            cf.launch = launch_condense<D, K, float>;
          }
        else
          {
            cf.fn     = reinterpret_cast<const void *>(condense3_kernel<D, K, double>);
            cf.launch = launch_condense<D, K, double>;
          }
        return true;
      }
    else
      {
        cf.fn     = reinterpret_cast<const void *>(condense2_kernel<D, K>);
        cf.launch = launch_condense<D, K, double>;
        return !mixed;
      }
  }

  bool
  kernels_for(int dim, int k, CondenseKernel &cf, ReconstructFn &rf, bool mixed = false)
  {
    switch (dim * 10 + k)
      {
        case 11: return pick<1, 1>(cf, rf, mixed);
        case 12: return pick<1, 2>(cf, rf, mixed);
        case 13: return pick<1, 3>(cf, rf, mixed);
        case 21: return pick<2, 1>(cf, rf, mixed);
        case 22: return pick<2, 2>(cf, rf, mixed);
        case 23: return pick<2, 3>(cf, rf, mixed);
        case 31: return pick<3, 1>(cf, rf, mixed);
        case 32: return pick<3, 2>(cf, rf, mixed);
        default: return false;
      }
  }

  // table staging and placement of the right-hand-side block R so that one
  // cell's workspace (one CTA of CondenseTPB threads) fits in the 227 KB of
  // shared memory of a CTA; R moves to global memory only when nothing else
  // makes it fit
  int
  launch_shape(const ddhdg_ctx *c, const Mode &m, int &stage, bool &r_global, size_t &smem)
  {
    const size_t limit = 220 * 1024;
    const size_t tb    = (((size_t)c->to.total + 1) & ~(size_t)1) * sizeof(double);
    for (int rg = 0; rg < 2; ++rg)
      for (stage = 1; stage >= 0; --stage)
        {
          r_global       = rg != 0;
          const Ws2Off w = ws2_layout(c->dim, c->nb, c->nf, m.ncomp, m.ncol, r_global);
          smem           = (stage ? tb : 0) + (size_t)w.total * sizeof(double);
          if (smem <= limit)
            return DDHDG_OK;
        }
    return fail(DDHDG_BAD_ARG, "the per-cell workspace does not fit in shared memory");
  }

  __global__ void
  scatter_kernel(int64_t ncells, int F, int nf, int ncomp, int Nt, const double *tt,
                 const double *rhs, const int32_t *dflag, const double *dval,
                 const uint8_t *slots, const int32_t *rowptr, double *csr,
                 double *grhs, int n0, int n1, const int64_t fo0, const int64_t fo1,
                 const int64_t fo2, int e00, int e01, int e02, int e10, int e11,
                 int e12, int e20, int e21, int e22, int dim)
  {
    const int64_t tot = ncells * (int64_t)Nt * Nt;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < tot;
         idx += (int64_t)gridDim.x * blockDim.x)
      {
        const int64_t cell = idx / ((int64_t)Nt * Nt);
        const int     i    = (int)((idx / Nt) % Nt);
        const int     j    = (int)(idx % Nt);
        const int     fi = i / (ncomp * nf), fj = j / (ncomp * nf);
        int ci[3];
        ci[0] = (int)(cell % n0);
        ci[1] = (int)((cell / n0) % n1);
        ci[2] = (int)(cell / ((int64_t)n0 * n1));
        const int64_t off[3] = {fo0, fo1, fo2};
        const int     ext[3][3] = {{e00, e01, e02}, {e10, e11, e12}, {e20, e21, e22}};
        int           cf[3] = {ci[0], ci[1], ci[2]};
        const int     a     = fi / 2;
        cf[a] += fi % 2;
        int64_t fidx = 0, stride = 1;
        for (int b = 0; b < dim; ++b)
          {
            fidx += cf[b] * stride;
            stride *= ext[a][b];
          }
        const int64_t Fi  = off[a] + fidx;
        const int64_t row = Fi * ncomp * nf + (i % (ncomp * nf));
        const int     sl  = slots[(cell * F + fi) * F + fj];
        const int64_t pos = rowptr[row] + (int64_t)sl * ncomp * nf + (j % (ncomp * nf));
        const double  v   = tt[idx];
        if (v != 0.)
          atomicAdd(csr + pos, v);
        if (j == i && dflag[cell * Nt + i])
          {
            atomicAdd(csr + pos, 1.);
            atomicAdd(grhs + row, dval[cell * Nt + i]);
          }
        else if (j == 0 && !dflag[cell * Nt + i])
          atomicAdd(grhs + row, rhs[cell * Nt + i]);
      }
  }

  // scale row i of a CSR system (values and rhs) by 1 / max_j |a_ij|
  __global__ void
  row_equilibrate_kernel(int64_t n, const int32_t *rowptr, double *val, double *rhs)
  {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
      {
        double mx = 0.;
        for (int32_t k = rowptr[i]; k < rowptr[i + 1]; ++k)
          mx = fmax(mx, fabs(val[k]));
        if (mx > 0.)
          {
            const double sc = 1. / mx;
            for (int32_t k = rowptr[i]; k < rowptr[i + 1]; ++k)
              val[k] *= sc;
            rhs[i] *= sc;
          }
      }
  }

  __global__ void
  gather_kernel(int64_t n, const int32_t *map, const double *src, double *dst)
  {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
      dst[i] = src[map[i]];
  }

  __global__ void
  scatter_perm_kernel(int64_t n, const int32_t *perm, const double *src, double *dst)
  {
    // dst[perm[i]] = src[i]
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
      dst[perm[i]] = src[i];
  }

  // restricted solution -> full trace update [nfaces][3][nf]
  __global__ void
  expand_kernel(int64_t nfaces, int nf, int ncomp, int c0, int c1, int c2,
                const double *x, double *full)
  {
    const int     comps[3] = {c0, c1, c2};
    const int64_t tot      = nfaces * 3 * nf;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < tot;
         i += (int64_t)gridDim.x * blockDim.x)
      {
        const int64_t f = i / (3 * nf);
        const int     b = (int)((i / nf) % 3);
        const int     m = (int)(i % nf);
        int           ce = -1;
        for (int c = 0; c < ncomp; ++c)
          if (comps[c] == b)
            ce = c;
        full[i] = (ce >= 0) ? x[(f * ncomp + ce) * nf + m] : 0.;
      }
  }

  // out[0] = max|a|, out[1] = max|b|, out[2] = max|c|, out[3] = max|d|
  __global__ void
  absmax_kernel(const double *a, int64_t na, const double *b, int64_t nb_,
                const double *c, int64_t nc, const double *d, int64_t nd,
                unsigned long long *out)
  {
    double m[4] = {0., 0., 0., 0.};
    const double *arr[4] = {a, b, c, d};
    const int64_t n[4]   = {na, nb_, nc, nd};
    for (int k = 0; k < 4; ++k)
      for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n[k];
           i += (int64_t)gridDim.x * blockDim.x)
        {
          const double v = fabs(arr[k][i]);
          m[k]           = (v > m[k] || v != v) ? v : m[k];
        }
    for (int k = 0; k < 4; ++k)
      {
        double v = m[k];
        for (int o = 16; o > 0; o >>= 1)
          {
            const double w = __shfl_xor_sync(0xffffffffu, v, o);
            v              = (w != w || w > v) ? w : v; // keeps NaN
          }
        if ((threadIdx.x & 31) == 0)
          atomicMax(out + k, __double_as_longlong(v));
      }
  }

  __global__ void
  axpy2_kernel(int64_t n1, double *y1, const double *x1, int64_t n2, double *y2,
               const double *x2, double alpha)
  {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n1 + n2;
         i += (int64_t)gridDim.x * blockDim.x)
      {
        if (i < n1)
          y1[i] += alpha * x1[i];
        else
          y2[i - n1] += alpha * x2[i - n1];
      }
  }

  // L2 projection of point values into the scalar + weak-gradient flux
  // coefficients of one component (src/project_component.cpp:268-420).
  // mode 0: values given; mode 1: density of comp from the quasi Fermi
  // potential qf and the cell's V (include/solver.h:378-412).
  __global__ void
  project_cell_kernel(int64_t ncells, int dim, int nb, int nqc, int nqf, int F,
                      const double *tab, TabOff to, const double *vc, const double *vf,
                      int comp, double *cell_state, int mode, double qf_pot,
                      double T, double V_rescale, double n_rescale, double nband,
                      double eband)
  {
    const double *phi_c  = tab + to.phi_c;
    const double *grad_c = tab + to.grad_c;
    const double *w_c    = tab + to.w_c;
    const double *phi_f  = tab + to.phi_f;
    const double *w_f    = tab + to.w_f;
    const double *minv   = tab + to.minv;
    const int     NCA    = 3 * (dim + 1) * nb;
    for (int64_t cell = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; cell < ncells;
         cell += (int64_t)gridDim.x * blockDim.x)
      {
        double       *cs = cell_state + cell * NCA;
        const double *Vs = cs + (0 * (dim + 1) + dim) * nb;
        double        rc[64], rd[3][64], val[64], valf[6][16];
        for (int q = 0; q < nqc; ++q)
          {
            double v;
            if (mode == 0)
              v = vc[cell * nqc + q];
            else
              {
                double V = 0.;
                for (int a = 0; a < nb; ++a)
                  V += phi_c[q * nb + a] * Vs[a];
                V *= V_rescale;
                const double kT = KB_ * T;
                const double ex = (comp == 1) ? (Q_ * (V - qf_pot) - eband) / kT :
                                                (Q_ * (qf_pot - V) + eband) / kT;
                v               = nband * exp(ex) / n_rescale;
              }
            val[q] = v;
          }
        for (int f = 0; f < F; ++f)
          for (int q = 0; q < nqf; ++q)
            {
              double v;
              if (mode == 0)
                v = vf[(cell * F + f) * nqf + q];
              else
                {
                  double V = 0.;
                  for (int a = 0; a < nb; ++a)
                    V += phi_f[(f * nqf + q) * nb + a] * Vs[a];
                  V *= V_rescale;
                  const double kT = KB_ * T;
                  const double ex = (comp == 1) ? (Q_ * (V - qf_pot) - eband) / kT :
                                                  (Q_ * (qf_pot - V) + eband) / kT;
                  v               = nband * exp(ex) / n_rescale;
                }
              valf[f][q] = v;
            }
        for (int b = 0; b < nb; ++b)
          {
            double acc = 0.;
            for (int q = 0; q < nqc; ++q)
              acc += w_c[q] * phi_c[q * nb + b] * val[q];
            rc[b] = acc;
            for (int s = 0; s < dim; ++s)
              {
                double ad = 0.;
                for (int q = 0; q < nqc; ++q)
                  ad += w_c[q] * grad_c[(q * nb + b) * dim + s] * val[q];
                for (int f = 0; f < F; ++f)
                  {
                    if (f / 2 != s)
                      continue;
                    const double ns = (f & 1) ? 1. : -1.;
                    for (int q = 0; q < nqf; ++q)
                      ad -= ns * w_f[f * nqf + q] * phi_f[(f * nqf + q) * nb + b] * valf[f][q];
                  }
                rd[s][b] = ad;
              }
          }
        double *blk = cs + comp * (dim + 1) * nb;
        for (int a = 0; a < nb; ++a)
          {
            double u = 0.;
            for (int b = 0; b < nb; ++b)
              u += minv[a * nb + b] * rc[b];
            blk[dim * nb + a] = u;
            for (int s = 0; s < dim; ++s)
              {
                double w = 0.;
                for (int b = 0; b < nb; ++b)
                  w += minv[a * nb + b] * rd[s][b];
                blk[s * nb + a] = w;
              }
          }
      }
  }

  // L2 projection of face point values on the trace of comp.  mode 0:
  // values [nfaces][nqf]; mode 1: l2_average of the two cells' values of comp
  // (src/copy_on_trace.cpp:631-1010 with c_strategy 0).
  __global__ void
  project_trace_kernel(int64_t nfaces, int dim, int nb, int nf, int nqf, int F,
                       const double *tab, TabOff to, const double *vals, int comp,
                       double *trace_state, int mode, const double *cell_state,
                       const int64_t *face_cells, const int64_t *cell_face_local)
  {
    const double *phi_f  = tab + to.phi_f;
    const double *fminvw = tab + to.fminvw;
    const int     NCA    = 3 * (dim + 1) * nb;
    for (int64_t Fi = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; Fi < nfaces;
         Fi += (int64_t)gridDim.x * blockDim.x)
      {
        double v[16];
        for (int q = 0; q < nqf; ++q)
          v[q] = 0.;
        if (mode == 0)
          for (int q = 0; q < nqf; ++q)
            v[q] = vals[Fi * nqf + q];
        else
          {
            int cnt = 0;
            for (int sd = 0; sd < 2; ++sd)
              {
                const int64_t cell = face_cells[Fi * 2 + sd];
                if (cell < 0)
                  continue;
                ++cnt;
                const int     f  = (int)cell_face_local[Fi * 2 + sd];
                const double *cs = cell_state + cell * NCA + (comp * (dim + 1) + dim) * nb;
                for (int q = 0; q < nqf; ++q)
                  {
                    double u = 0.;
                    for (int a = 0; a < nb; ++a)
                      u += phi_f[(f * nqf + q) * nb + a] * cs[a];
                    v[q] += u;
                  }
              }
            for (int q = 0; q < nqf; ++q)
              v[q] /= cnt;
          }
        for (int m = 0; m < nf; ++m)
          {
            double acc = 0.;
            for (int q = 0; q < nqf; ++q)
              acc += fminvw[m * nqf + q] * v[q];
            trace_state[(Fi * 3 + comp) * nf + m] = acc;
          }
      }
  }

  int
  grid_for(const ddhdg_ctx *c, int64_t work, int block);

  // the context's nested-dissection trace solver for one mode (built on
  // first use: symbolic phase on the host, fronts on the device)
  int
  nd_solver(ddhdg_ctx *c, Mode &m, NDSolver *&out)
  {
    if (!m.nd)
      {
        NDSolver::Mesh M;
        M.dim = c->dim;
        for (int a = 0; a < 3; ++a)
          {
            M.n[a]        = (a < c->dim) ? c->desc.n[a] : 1;
            M.face_off[a] = c->face_off[a];
            for (int b = 0; b < 3; ++b)
              M.face_ext[a][b] = c->face_ext[a][b];
          }
        M.ncells = c->ncells;
        M.nfaces = c->nfaces;
        M.F      = c->F;
        M.nd     = m.ncomp * c->nf;
        std::unique_ptr<NDSolver> nd(new NDSolver);
        std::string               err;
        const int                 r = nd->build(M, err);
        if (r)
          return fail(r, err);
        nd->set_graphs(c->solver_graphs);
        m.nd = std::move(nd);
      }
    out = m.nd.get();
    return DDHDG_OK;
  }

  int
  grid_for(const ddhdg_ctx *c, int64_t work, int block)
  {
    int64_t g = (work + block - 1) / block;
    g         = std::min<int64_t>(g, (int64_t)c->sm_count * 32);
    return (int)std::max<int64_t>(g, 1);
  }
} // namespace

extern "C" {

const char *
ddhdg_last_error(void)
{
  return g_last_error.c_str();
}

int
ddhdg_reference_points(int dim, int degree, double *qref_c, double *qref_f, double *support)
{
  if (dim < 1 || dim > 3 || degree < 0 || degree > 6)
    return fail(DDHDG_BAD_ARG, "bad dim/degree");
  const double h[3] = {1., 1., 1.};
  const Tables T    = build_tables(dim, degree, h);
  if (qref_c)
    std::copy(T.qref_c.begin(), T.qref_c.end(), qref_c);
  if (qref_f)
    std::copy(T.qref_f.begin(), T.qref_f.end(), qref_f);
  if (support)
    std::copy(T.gl.begin(), T.gl.end(), support);
  return DDHDG_OK;
}

int
ddhdg_ctx_create(const ddhdg_problem_desc *d, ddhdg_ctx **out)
{
  if (!d || !out)
    return fail(DDHDG_BAD_ARG, "null argument");
  *out = nullptr;
  if (d->dim < 1 || d->dim > 3 || d->degree < 1 || d->degree > 3)
    return fail(DDHDG_BAD_ARG, "dim must be 1..3 and degree 1..3");
  if (d->dim == 3 && d->degree > 2)
    return fail(DDHDG_BAD_ARG, "3D supports degree 1 and 2");
  if (d->precision != 0 && d->precision != 1)
    return fail(DDHDG_BAD_ARG, "precision must be 0 (FP64) or 1 (mixed)");
  {
    int nb = 1;
    for (int a = 0; a < d->dim; ++a)
      nb *= d->degree + 1;
    if (d->precision == 1 && 3 * nb > 32)
      return fail(DDHDG_BAD_ARG, "mixed precision needs 3 (k+1)^d <= 32 (1D, 2D k <= 2, 3D k = 1)");
  }
  {
    int64_t cells = 1;
    for (int a = 0; a < d->dim; ++a)
      {
        if (d->n[a] < 1 || !(d->h[a] > 0.))
          return fail(DDHDG_BAD_ARG, "bad mesh");
        cells *= d->n[a];
        if (cells >= (int64_t(1) << 31))
          return fail(DDHDG_BAD_ARG, "a context holds fewer than 2^31 cells");
      }
  }
  if (!d->doping_host || !d->face_bc_host || !d->face_bc_val_host)
    return fail(DDHDG_BAD_ARG, "doping and boundary tables are required");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    {
      cudaGetLastError();
      return fail(DDHDG_NO_DEVICE, "no CUDA device");
    }
  auto c  = std::make_unique<ddhdg_ctx>();
  c->desc = *d;
  c->dim  = d->dim;
  c->k    = d->degree;
  c->T    = build_tables(d->dim, d->degree, d->h);
  {
    const double unit[3] = {1., 1., 1.};
    c->Tu                = build_tables(d->dim, d->degree, unit);
  }
  c->nb   = c->T.nb;
  c->nf   = c->T.nf;
  c->nqc  = c->T.nqc;
  c->nqf  = c->T.nqf;
  c->F    = c->T.F;
  for (int b = 0; b < 3; ++b)
    c->enabled[b] = d->enabled[b] ? 1 : 0;
  c->ncells = 1;
  for (int a = 0; a < d->dim; ++a)
    c->ncells *= d->n[a];
  int64_t off = 0;
  for (int a = 0; a < d->dim; ++a)
    {
      c->face_off[a] = off;
      int64_t cnt    = 1;
      for (int b = 0; b < 3; ++b)
        {
          const int e      = (b < d->dim) ? (d->n[b] + (b == a ? 1 : 0)) : 1;
          c->face_ext[a][b] = e;
          cnt *= e;
        }
      off += cnt;
    }
  c->nfaces = off;
  // face -> cells
  c->face_cells.assign(c->nfaces * 2, -1);
  for (int64_t cell = 0; cell < c->ncells; ++cell)
    for (int f = 0; f < c->F; ++f)
      {
        const int64_t Fi            = face_of_cell(c.get(), cell, f);
        c->face_cells[Fi * 2 + (1 - f % 2)] = cell;
      }
  {
    std::vector<int64_t> loc(c->nfaces * 2, -1);
    for (int64_t cell = 0; cell < c->ncells; ++cell)
      for (int f = 0; f < c->F; ++f)
        loc[face_of_cell(c.get(), cell, f) * 2 + (1 - f % 2)] = f;
    int r0;
    if ((r0 = c->d_face_cells.upload(c->face_cells.data(), c->face_cells.size())))
      return r0;
    if ((r0 = c->d_face_local.upload(loc.data(), loc.size())))
      return r0;
  }
  // stage the tables in one block
  {
    std::vector<double> blob;
    auto put = [&](const std::vector<double> &v) {
      int o = (int)blob.size();
      blob.insert(blob.end(), v.begin(), v.end());
      while (blob.size() % 2)
        blob.push_back(0.);
      return o;
    };
    c->to.phi_c  = put(c->T.phi_c);
    c->to.grad_c = put(c->T.grad_c);
    c->to.w_c    = put(c->T.w_c);
    c->to.phi_f  = put(c->T.phi_f);
    c->to.w_f    = put(c->T.w_f);
    c->to.xi     = put(c->T.xi);
    c->to.fminvw = put(c->T.fminvw);
    c->to.PW_c   = put(c->T.PW_c);
    c->to.PW_f   = put(c->T.PW_f);
    c->to.QW_c   = put(c->T.QW_c);
    c->to.QW_f   = put(c->T.QW_f);
    c->to.P      = put(c->T.P);
    c->to.Q      = put(c->T.Q);
    c->to.minv   = put(c->T.minv);
    c->to.TLc    = put(c->T.TLc);
    c->to.TLg    = put(c->T.TLg);
    c->to.TLf    = put(c->T.TLf);
    c->to.RTk    = put(c->T.RTk);
    c->to.RTr    = put(c->T.RTr);
    c->to.RQk    = put(c->T.RQk);
    c->to.RQr    = put(c->T.RQr);
    c->to.total  = (int)blob.size();
    int r        = c->tables.upload(blob.data(), blob.size());
    if (r)
      return r;
  }
  int r;
  const int64_t nq = c->ncells * c->nqc;
  if ((r = c->doping.upload(d->doping_host, nq)))
    return r;
  if (d->rec_a_host && (r = c->rec_a.upload(d->rec_a_host, nq)))
    return r;
  if (d->rec_b_host && (r = c->rec_b.upload(d->rec_b_host, nq)))
    return r;
  if (d->rec_c_host && (r = c->rec_c.upload(d->rec_c_host, nq)))
    return r;
  if (d->tau_host && (r = c->tau_table.upload(d->tau_host, c->ncells * c->F * 3)))
    return r;
  if ((r = c->bc.upload(d->face_bc_host, c->nfaces * 3)))
    return r;
  if ((r = c->bc_val.upload(d->face_bc_val_host, c->nfaces * 3 * c->nqf)))
    return r;
  if ((r = c->status.alloc(1)))
    return r;
  CK(cudaMemset(c->status.p, 0, sizeof(int)));
  int dev = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, dev));
  // host pointers are not kept
  c->desc.doping_host = nullptr;
  c->desc.rec_a_host = c->desc.rec_b_host = c->desc.rec_c_host = nullptr;
  c->desc.tau_host                                             = nullptr;
  c->desc.face_bc_host                                         = nullptr;
  c->desc.face_bc_val_host                                     = nullptr;
  *out = c.release();
  return DDHDG_OK;
}

int
ddhdg_ctx_destroy(ddhdg_ctx *c)
{
  if (!c)
    return DDHDG_OK;
  if (c->sp)
    cusolverSpDestroy(c->sp);
  if (c->descr)
    cusparseDestroyMatDescr(c->descr);
  delete c;
  return DDHDG_OK;
}

int
ddhdg_get_sizes(const ddhdg_ctx *cc, int thermo, ddhdg_sizes *s)
{
  if (!cc || !s)
    return fail(DDHDG_BAD_ARG, "null argument");
  ddhdg_ctx *c = const_cast<ddhdg_ctx *>(cc);
  thermo       = thermo ? 1 : 0;
  int r;
  if (!c->mode[thermo].built && (r = build_mode(c, thermo)))
    return r;
  const Mode &m  = c->mode[thermo];
  s->ncells      = c->ncells;
  s->nfaces      = c->nfaces;
  s->Nc_all      = 3 * (c->dim + 1) * c->nb;
  s->Nt          = m.Nt;
  s->ncomp       = m.ncomp;
  s->nqc         = c->nqc;
  s->nqf         = c->nqf;
  s->nb          = c->nb;
  s->nf          = c->nf;
  s->n_trace_dofs = m.ndofs;
  s->nnz         = m.nnz;
  return DDHDG_OK;
}

int
ddhdg_set_boundary(ddhdg_ctx *c, const int32_t *bc, const double *val)
{
  if (!c || !bc || !val)
    return fail(DDHDG_BAD_ARG, "null argument");
  int r;
  if ((r = c->bc.upload(bc, c->nfaces * 3)))
    return r;
  return c->bc_val.upload(val, c->nfaces * 3 * c->nqf);
}

int
ddhdg_set_enabled(ddhdg_ctx *c, int V, int n, int p)
{
  if (!c)
    return fail(DDHDG_BAD_ARG, "null argument");
  if (!V && !n && !p)
    return fail(DDHDG_BAD_ARG, "no component enabled");
  const int nv[3] = {V ? 1 : 0, n ? 1 : 0, p ? 1 : 0};
  if (nv[0] != c->enabled[0] || nv[1] != c->enabled[1] || nv[2] != c->enabled[2])
    {
      for (int b = 0; b < 3; ++b)
        c->enabled[b] = nv[b];
      c->mode[0].built = false;
    }
  return DDHDG_OK;
}

// the condense launch over the cells [c0, c1)
static int
condense_range(ddhdg_ctx *c, const double *cell_state, const double *trace_state, int thermo,
               double *tt, double *rhs, int32_t *dflag, double *dval, ddhdg_stream_t stream,
               int64_t c0, int64_t c1)
{
  if (!c || !cell_state || !trace_state || !tt || !rhs || !dflag || !dval)
    return fail(DDHDG_BAD_ARG, "null argument");
  thermo = thermo ? 1 : 0;
  int r;
  if ((r = ensure_buffers(c, thermo)))
    return r;
  Mode      &m = c->mode[thermo];
  CondenseKernel cf;
  ReconstructFn rf;
  const bool mixed = c->desc.precision == 1;
  if (!kernels_for(c->dim, c->k, cf, rf, mixed))
    return fail(DDHDG_BAD_ARG, "unsupported dim/degree");
  KParams P     = make_params(c, thermo);
  P.cell0       = c0;
  P.ncells      = c1;
  P.cell_state  = cell_state;
  P.trace_state = trace_state;
  P.tt          = tt;
  P.rhs         = rhs;
  P.dflag       = dflag;
  P.dval        = dval;
  P.ycache      = m.ycache.p;
  int    threads;
  size_t smem;
  int64_t units;
  if (3 * c->nb <= 32)
    {
      // warp per cell: as many warps per CTA as shared memory allows
      // mixed: two CTAs per SM (the FP32 kernel is built for 128 registers)
      const Ws3Off w   = ws3_layout(c->dim, c->nb, c->nf, m.ncomp, m.ncol, mixed ? 4 : 8);
      const size_t per = (size_t)w.total * sizeof(double);
      int          wpb = (int)std::min<size_t>(Condense3MaxWPB, (mixed ? 110 : 220) * 1024 / per);
      if (wpb < 1)
        return fail(DDHDG_BAD_ARG, "the per-cell workspace does not fit in shared memory");
      P.wpb   = wpb;
      P.stage = 0;
      threads = wpb * 32;
      smem    = (size_t)wpb * per;
      units   = (c1 - c0 + wpb - 1) / wpb;
    }
  else
    {
      int  stage;
      bool r_global;
      if ((r = launch_shape(c, m, stage, r_global, smem)))
        return r;
      P.wpb   = 1;
      P.stage = stage;
      threads = CondenseTPB;
      units   = c1 - c0;
      if (r_global)
        {
          int per_sm = 0;
          CK(allow_full_dynamic_smem(cf.fn));
          CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, cf.fn, threads, smem));
          const int64_t g = std::min<int64_t>(units, (int64_t)std::max(per_sm, 1) * c->sm_count);
          if ((r = m.rscratch.alloc((size_t)g * c->nb * m.ncomp * m.ncol)))
            return r;
          P.rscratch = m.rscratch.p;
        }
    }
  CK(allow_full_dynamic_smem(cf.fn));
  int per_sm = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, cf.fn, threads, smem));
  if (per_sm < 1)
    return fail(DDHDG_BAD_ARG, "condense kernel does not fit on an SM");
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(units, (int64_t)per_sm * c->sm_count));
  cf.launch(c->Tu, P, grid, threads, smem, (cudaStream_t)stream);
  CK(cudaGetLastError());
  return DDHDG_OK;
}

int
ddhdg_assemble_condense(ddhdg_ctx *c, const double *cell_state,
                        const double *trace_state, int thermo, double *tt,
                        double *rhs, int32_t *dflag, double *dval,
                        ddhdg_stream_t stream)
{
  if (!c)
    return fail(DDHDG_BAD_ARG, "null argument");
  return condense_range(c, cell_state, trace_state, thermo, tt, rhs, dflag, dval, stream, 0, c->ncells);
}

int
ddhdg_solve_condensed(ddhdg_ctx *c, const double *tt, const double *rhs, const int32_t *dflag,
                      const double *dval, double *x, int thermo, ddhdg_stream_t stream)
{
  if (!c || !tt || !rhs || !dflag || !dval || !x)
    return fail(DDHDG_BAD_ARG, "null argument");
  thermo = thermo ? 1 : 0;
  int   r;
  Mode &m = c->mode[thermo];
  if (!m.built && (r = build_mode(c, thermo)))
    return r;
  NDSolver *nd = nullptr;
  if ((r = nd_solver(c, m, nd)))
    return r;
  std::string err;
  if ((r = nd->solve(tt, rhs, dflag, dval, m.Nt, x, (cudaStream_t)stream, c->sm_count, err)))
    return fail(r, err);
  return DDHDG_OK;
}

int
ddhdg_trace_solver_bytes(int dim, const int *n, int degree, int ncomp, int64_t *bytes)
{
  if (!n || !bytes)
    return fail(DDHDG_BAD_ARG, "null argument");
  if (dim < 1 || dim > 3 || degree < 1 || degree > 3 || ncomp < 1 || ncomp > 3)
    return fail(DDHDG_BAD_ARG, "dim 1-3, degree 1-3 and 1-3 components");
  NDSolver::Mesh M;
  M.dim    = dim;
  M.ncells = 1;
  int nf   = 1;
  for (int a = 0; a < dim; ++a)
    {
      if (n[a] < 1)
        return fail(DDHDG_BAD_ARG, "bad mesh");
      M.n[a] = n[a];
      M.ncells *= n[a];
      if (a > 0)
        nf *= degree + 1;
    }
  // the faces in the layout of ddhdg_ctx_create: direction by direction
  int64_t off = 0;
  for (int a = 0; a < dim; ++a)
    {
      M.face_off[a] = off;
      int64_t cnt   = 1;
      for (int b = 0; b < 3; ++b)
        {
          const int e       = (b < dim) ? (n[b] + (b == a ? 1 : 0)) : 1;
          M.face_ext[a][b] = e;
          cnt *= e;
        }
      off += cnt;
    }
  M.nfaces = off;
  M.F      = 2 * dim;
  M.nd     = ncomp * nf;
  NDSolver    nd;
  std::string err;
  const int   r = nd.plan(M, err);
  if (r)
    return fail(r, err);
  *bytes = nd.planned_device_bytes();
  return DDHDG_OK;
}

int
ddhdg_release_solver(ddhdg_ctx *c, int thermo)
{
  if (!c)
    return fail(DDHDG_BAD_ARG, "null argument");
  c->mode[thermo ? 1 : 0].nd.reset();
  return DDHDG_OK;
}

int
ddhdg_set_solver_graphs(ddhdg_ctx *c, int enable)
{
  if (!c)
    return fail(DDHDG_BAD_ARG, "null argument");
  c->solver_graphs = enable != 0;
  for (auto &m : c->mode)
    if (m.nd)
      m.nd->set_graphs(c->solver_graphs);
  return DDHDG_OK;
}

// the reconstruction launch over the cells [c0, c1)
static int
reconstruct_range(ddhdg_ctx *c, const double *cell_state, const double *trace_state,
                  const double *update_trace, double *update_cell, int thermo,
                  ddhdg_stream_t stream, int64_t c0, int64_t c1)
{
  if (!c || !cell_state || !trace_state || !update_trace || !update_cell)
    return fail(DDHDG_BAD_ARG, "null argument");
  thermo = thermo ? 1 : 0;
  Mode &m = c->mode[thermo];
  if (!m.built || !m.ycache.p)
    return fail(DDHDG_BAD_ARG, "ddhdg_reconstruct needs a preceding ddhdg_assemble_condense");
  CondenseKernel cf;
  ReconstructFn rf;
  if (!kernels_for(c->dim, c->k, cf, rf))
    return fail(DDHDG_BAD_ARG, "unsupported dim/degree");
  KParams P     = make_params(c, thermo);
  P.cell0       = c0;
  P.ncells      = c1;
  P.cell_state  = cell_state;
  P.trace_state = trace_state;
  P.ycache      = m.ycache.p;
  const int    Ns  = m.ncomp * c->nb;
  const int    wsz = (Ns + 2 * c->F * 3 * c->nf + c->nb + m.Nt + 1) & ~1;
  const int    wpb = 8;
  const size_t nPQ = (size_t)(c->to.minv - c->to.P);
  const size_t smem =
    ((nPQ + 1) & ~(size_t)1) * sizeof(double) + (size_t)wpb * wsz * sizeof(double);
  P.wpb = wpb;
  CK(allow_full_dynamic_smem(reinterpret_cast<const void *>(rf)));
  int per_sm = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, rf, wpb * 32, smem));
  const int64_t blocks_needed = (c1 - c0 + wpb - 1) / wpb;
  const int     grid =
    (int)std::max<int64_t>(1, std::min<int64_t>(blocks_needed, (int64_t)std::max(per_sm, 1) * c->sm_count));
  rf<<<grid, wpb * 32, smem, (cudaStream_t)stream>>>(P, update_trace, update_cell);
  CK(cudaGetLastError());
  return DDHDG_OK;
}

int
ddhdg_reconstruct(ddhdg_ctx *c, const double *cell_state, const double *trace_state,
                  const double *update_trace, double *update_cell, int thermo,
                  ddhdg_stream_t stream)
{
  if (!c)
    return fail(DDHDG_BAD_ARG, "null argument");
  return reconstruct_range(c, cell_state, trace_state, update_trace, update_cell, thermo, stream, 0,
                           c->ncells);
}

// device copies, copy streams and events of the host-buffer calls (first use)
static int
hostio_setup(ddhdg_ctx *c)
{
  auto &h = c->hio;
  if (h.ready)
    return DDHDG_OK;
  const size_t ncell = (size_t)c->ncells * 3 * (c->dim + 1) * c->nb;
  const size_t ntr   = (size_t)c->nfaces * 3 * c->nf;
  int          r;
  if ((r = h.cell.alloc(ncell)) || (r = h.trace.alloc(ntr)) || (r = h.dtrace.alloc(ntr)) ||
      (r = h.dcell.alloc(ncell)))
    return r;
  CK(cudaStreamCreateWithFlags(&h.h2d, cudaStreamNonBlocking));
  CK(cudaStreamCreateWithFlags(&h.d2h, cudaStreamNonBlocking));
  for (cudaEvent_t *e : {&h.ev_trace, &h.ev_out, &h.ev_cell_free, &h.ev_dtrace_free})
    CK(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
  for (int k = 0; k < ddhdg_ctx::HostIO::NChunk; ++k)
    {
      CK(cudaEventCreateWithFlags(&h.ev_chunk[k], cudaEventDisableTiming));
      CK(cudaEventCreateWithFlags(&h.ev_rec[k], cudaEventDisableTiming));
    }
  h.ready = true;
  return DDHDG_OK;
}

static int64_t
hostio_chunk_begin(const ddhdg_ctx *c, int k)
{
  return c->ncells * k / ddhdg_ctx::HostIO::NChunk;
}

int
ddhdg_assemble_condense_host(ddhdg_ctx *c, const double *cell_state_host,
                             const double *trace_state_host, int thermo, double *tt, double *rhs,
                             int32_t *dflag, double *dval, ddhdg_stream_t stream)
{
  if (!c || !cell_state_host || !trace_state_host || !tt || !rhs || !dflag || !dval)
    return fail(DDHDG_BAD_ARG, "null argument");
  int r;
  if ((r = hostio_setup(c)))
    return r;
  auto        &h  = c->hio;
  cudaStream_t s  = (cudaStream_t)stream;
  const size_t pc = (size_t)3 * (c->dim + 1) * c->nb; // doubles per cell
  // the device copies are rewritten once the kernels that read them (the
  // previous condensation or reconstruction) are done
  CK(cudaStreamWaitEvent(h.h2d, h.ev_cell_free, 0));
  CK(cudaMemcpyAsync(h.trace.p, trace_state_host, (size_t)c->nfaces * 3 * c->nf * sizeof(double),
                     cudaMemcpyHostToDevice, h.h2d));
  CK(cudaEventRecord(h.ev_trace, h.h2d));
  for (int k = 0; k < ddhdg_ctx::HostIO::NChunk; ++k)
    {
      const int64_t c0 = hostio_chunk_begin(c, k), c1 = hostio_chunk_begin(c, k + 1);
      CK(cudaMemcpyAsync(h.cell.p + c0 * pc, cell_state_host + c0 * pc, (size_t)(c1 - c0) * pc * sizeof(double),
                         cudaMemcpyHostToDevice, h.h2d));
      CK(cudaEventRecord(h.ev_chunk[k], h.h2d));
    }
  CK(cudaStreamWaitEvent(s, h.ev_trace, 0));
  for (int k = 0; k < ddhdg_ctx::HostIO::NChunk; ++k)
    {
      const int64_t c0 = hostio_chunk_begin(c, k), c1 = hostio_chunk_begin(c, k + 1);
      CK(cudaStreamWaitEvent(s, h.ev_chunk[k], 0));
      if (c1 > c0 &&
          (r = condense_range(c, h.cell.p, h.trace.p, thermo, tt, rhs, dflag, dval, stream, c0, c1)))
        return r;
    }
  CK(cudaEventRecord(h.ev_cell_free, s));
  h.have_state = true;
  return DDHDG_OK;
}

int
ddhdg_reconstruct_host(ddhdg_ctx *c, const double *update_trace_host, int thermo,
                       double *update_cell_host, ddhdg_stream_t stream)
{
  if (!c || !update_trace_host || !update_cell_host)
    return fail(DDHDG_BAD_ARG, "null argument");
  auto &h = c->hio;
  if (!h.have_state)
    return fail(DDHDG_BAD_ARG, "ddhdg_reconstruct_host needs a preceding ddhdg_assemble_condense_host");
  cudaStream_t s  = (cudaStream_t)stream;
  const size_t pc = (size_t)3 * (c->dim + 1) * c->nb;
  int          r;
  // the upload of the trace update may overlap the condensation still running
  CK(cudaStreamWaitEvent(h.h2d, h.ev_dtrace_free, 0));
  CK(cudaMemcpyAsync(h.dtrace.p, update_trace_host, (size_t)c->nfaces * 3 * c->nf * sizeof(double),
                     cudaMemcpyHostToDevice, h.h2d));
  CK(cudaEventRecord(h.ev_trace, h.h2d));
  CK(cudaStreamWaitEvent(s, h.ev_trace, 0));
  for (int k = 0; k < ddhdg_ctx::HostIO::NChunk; ++k)
    {
      const int64_t c0 = hostio_chunk_begin(c, k), c1 = hostio_chunk_begin(c, k + 1);
      if (c1 <= c0)
        continue;
      if ((r = reconstruct_range(c, h.cell.p, h.trace.p, h.dtrace.p, h.dcell.p, thermo, stream, c0, c1)))
        return r;
      CK(cudaEventRecord(h.ev_rec[k], s));
      CK(cudaStreamWaitEvent(h.d2h, h.ev_rec[k], 0));
      CK(cudaMemcpyAsync(update_cell_host + c0 * pc, h.dcell.p + c0 * pc, (size_t)(c1 - c0) * pc * sizeof(double),
                         cudaMemcpyDeviceToHost, h.d2h));
    }
  CK(cudaEventRecord(h.ev_cell_free, s));
  CK(cudaEventRecord(h.ev_dtrace_free, s));
  CK(cudaEventRecord(h.ev_out, h.d2h));
  CK(cudaStreamWaitEvent(s, h.ev_out, 0));
  return DDHDG_OK;
}

int
ddhdg_get_csr(ddhdg_ctx *c, int thermo, const int32_t **row_ptr, const int32_t **col_idx)
{
  if (!c || !row_ptr || !col_idx)
    return fail(DDHDG_BAD_ARG, "null argument");
  thermo = thermo ? 1 : 0;
  int r;
  if (!c->mode[thermo].built && (r = build_mode(c, thermo)))
    return r;
  *row_ptr = c->mode[thermo].rowptr.p;
  *col_idx = c->mode[thermo].colind.p;
  return DDHDG_OK;
}

int
ddhdg_scatter(ddhdg_ctx *c, const double *tt, const double *rhs, const int32_t *dflag,
              const double *dval, double *csr, double *grhs, int thermo,
              ddhdg_stream_t stream)
{
  if (!c || !tt || !rhs || !dflag || !dval || !csr || !grhs)
    return fail(DDHDG_BAD_ARG, "null argument");
  thermo  = thermo ? 1 : 0;
  Mode &m = c->mode[thermo];
  int   r;
  if (!m.built && (r = build_mode(c, thermo)))
    return r;
  cudaStream_t s = (cudaStream_t)stream;
  CK(cudaMemsetAsync(csr, 0, m.nnz * sizeof(double), s));
  CK(cudaMemsetAsync(grhs, 0, m.ndofs * sizeof(double), s));
  const int64_t tot = c->ncells * (int64_t)m.Nt * m.Nt;
  scatter_kernel<<<grid_for(c, tot, 256), 256, 0, s>>>(
    c->ncells, c->F, c->nf, m.ncomp, m.Nt, tt, rhs, dflag, dval, m.slots.p,
    m.rowptr.p, csr, grhs, c->desc.n[0], c->dim > 1 ? c->desc.n[1] : 1,
    c->face_off[0], c->face_off[1], c->face_off[2], c->face_ext[0][0],
    c->face_ext[0][1], c->face_ext[0][2], c->face_ext[1][0], c->face_ext[1][1],
    c->face_ext[1][2], c->face_ext[2][0], c->face_ext[2][1], c->face_ext[2][2], c->dim);
  CK(cudaGetLastError());
  return DDHDG_OK;
}

int
ddhdg_solve_trace(ddhdg_ctx *c, const double *csr, const double *grhs, double *x,
                  int thermo, ddhdg_stream_t stream)
{
  if (!c || !csr || !grhs || !x)
    return fail(DDHDG_BAD_ARG, "null argument");
  thermo  = thermo ? 1 : 0;
  Mode &m = c->mode[thermo];
  if (!m.built)
    return fail(DDHDG_BAD_ARG, "sparsity not built");
  cudaStream_t s = (cudaStream_t)stream;
  if (!c->sp)
    {
      if (cusolverSpCreate(&c->sp) != CUSOLVER_STATUS_SUCCESS)
        return fail(DDHDG_SOLVER_ERROR, "cusolverSpCreate failed");
      if (cusparseCreateMatDescr(&c->descr) != CUSPARSE_STATUS_SUCCESS)
        return fail(DDHDG_SOLVER_ERROR, "cusparseCreateMatDescr failed");
      cusparseSetMatType(c->descr, CUSPARSE_MATRIX_TYPE_GENERAL);
      cusparseSetMatIndexBase(c->descr, CUSPARSE_INDEX_BASE_ZERO);
    }
  cusolverSpSetStream(c->sp, s);
  int r;
  if ((r = m.pval.alloc(m.nnz)) || (r = m.pb.alloc(m.ndofs)) || (r = m.px.alloc(m.ndofs)))
    return r;
  // B = A(perm, perm), pb = b(perm)
  gather_kernel<<<grid_for(c, m.nnz, 256), 256, 0, s>>>(m.nnz, m.pmap.p, csr, m.pval.p);
  gather_kernel<<<grid_for(c, m.ndofs, 256), 256, 0, s>>>(m.ndofs, m.d_perm.p, grhs, m.pb.p);
  CK(cudaGetLastError());
  // Row equilibration: the potential rows are ~1e19 next to unit Dirichlet
  // identity rows, and Householder QR is only normwise backward stable, so
  // every row is scaled to max |a_ij| = 1 before the factorisation.
  row_equilibrate_kernel<<<grid_for(c, m.ndofs, 128), 128, 0, s>>>(m.ndofs, m.prow.p, m.pval.p, m.pb.p);
  CK(cudaGetLastError());
  int sing = -1;
  const cusolverStatus_t st = cusolverSpDcsrlsvqr(
    c->sp, (int)m.ndofs, (int)m.nnz, c->descr, m.pval.p, m.prow.p, m.pcol.p, m.pb.p,
    0.0, 0, m.px.p, &sing); // tol 0: only an exactly zero R diagonal counts as singular
  if (st != CUSOLVER_STATUS_SUCCESS)
    return fail(DDHDG_SOLVER_ERROR, "cusolverSpDcsrlsvqr failed with status " + std::to_string((int)st));
  if (sing >= 0)
    return fail(DDHDG_SOLVER_ERROR, "global trace matrix is singular at row " + std::to_string(sing));
  // x = px(iperm): x[perm[i]] = px[i]
  scatter_perm_kernel<<<grid_for(c, m.ndofs, 256), 256, 0, s>>>(m.ndofs, m.d_perm.p, m.px.p, x);
  CK(cudaGetLastError());
  return DDHDG_OK;
}

int
ddhdg_newton(ddhdg_ctx *c, double *cell_state, double *trace_state, int thermo,
             double abs_tol, double rel_tol, int max_it, double alpha, int *iterations,
             double *last_update_norm, ddhdg_stream_t stream)
{
  if (!c || !cell_state || !trace_state)
    return fail(DDHDG_BAD_ARG, "null argument");
  thermo = thermo ? 1 : 0;
  int r;
  if ((r = ensure_buffers(c, thermo)))
    return r;
  Mode         &m       = c->mode[thermo];
  cudaStream_t  s       = (cudaStream_t)stream;
  const int64_t ncell_d = c->ncells * 3 * (c->dim + 1) * c->nb;
  const int64_t ntr_d   = c->nfaces * 3 * c->nf;
  if ((r = m.csr.alloc(m.nnz)) || (r = m.grhs.alloc(m.ndofs)) || (r = m.x.alloc(m.ndofs)) ||
      (r = m.dtrace.alloc(ntr_d)) || (r = m.dcell.alloc(ncell_d)) ||
      (r = c->norm_buf.alloc(4)))
    return r;
  cudaEvent_t ev[4];
  for (auto &e : ev)
    CK(cudaEventCreate(&e));
  c->t_condense = c->t_solve = c->t_recon = 0.;
  c->t_steps                              = 0;
  bool   converged                        = false;
  int    step                             = 0;
  double upd_cell_norm                    = 0.;
  CK(cudaMemsetAsync(c->status.p, 0, sizeof(int), s));
  int rc = DDHDG_OK;
  while (max_it < 0 || step < max_it)
    {
      ++step;
      CK(cudaEventRecord(ev[0], s));
      if ((rc = ddhdg_assemble_condense(c, cell_state, trace_state, thermo, m.tt.p, m.rhs.p,
                                        m.dflag.p, m.dval.p, stream)))
        break;
      CK(cudaEventRecord(ev[1], s));
      if ((rc = ddhdg_solve_condensed(c, m.tt.p, m.rhs.p, m.dflag.p, m.dval.p, m.x.p, thermo,
                                      stream)))
        break;
      expand_kernel<<<grid_for(c, ntr_d, 256), 256, 0, s>>>(
        c->nfaces, c->nf, m.ncomp, m.comps[0], m.comps[1], m.comps[2], m.x.p, m.dtrace.p);
      CK(cudaEventRecord(ev[2], s));
      if ((rc = ddhdg_reconstruct(c, cell_state, trace_state, m.dtrace.p, m.dcell.p, thermo,
                                  stream)))
        break;
      CK(cudaEventRecord(ev[3], s));
      // norms: |dcell|, |dtrace|, |cell|, |trace| (before the update)
      CK(cudaMemsetAsync(c->norm_buf.p, 0, 4 * sizeof(double), s));
      absmax_kernel<<<grid_for(c, ncell_d, 256), 256, 0, s>>>(
        m.dcell.p, ncell_d, m.dtrace.p, ntr_d, cell_state, ncell_d, trace_state, ntr_d,
        reinterpret_cast<unsigned long long *>(c->norm_buf.p));
      axpy2_kernel<<<grid_for(c, ncell_d + ntr_d, 256), 256, 0, s>>>(
        ntr_d, trace_state, m.dtrace.p, ncell_d, cell_state, m.dcell.p, alpha);
      CK(cudaGetLastError());
      double nrm[4];
      int    status = 0;
      CK(cudaMemcpyAsync(nrm, c->norm_buf.p, 4 * sizeof(double), cudaMemcpyDeviceToHost, s));
      CK(cudaMemcpyAsync(&status, c->status.p, sizeof(int), cudaMemcpyDeviceToHost, s));
      CK(cudaStreamSynchronize(s));
      float t01, t12, t23;
      cudaEventElapsedTime(&t01, ev[0], ev[1]);
      cudaEventElapsedTime(&t12, ev[1], ev[2]);
      cudaEventElapsedTime(&t23, ev[2], ev[3]);
      c->t_condense += t01;
      c->t_solve += t12;
      c->t_recon += t23;
      c->t_steps += 1;
      if (status)
        {
          rc = fail(status, "a local cell system had a zero or non-finite pivot");
          break;
        }
      upd_cell_norm            = nrm[0];
      const double update_norm = std::max(nrm[0], nrm[1]);
      const double cur_norm    = std::max(nrm[2], nrm[3]);
      if (!std::isfinite(update_norm))
        {
          rc = fail(DDHDG_NOT_CONVERGED, "non-finite Newton update");
          break;
        }
      if (update_norm < abs_tol || update_norm < rel_tol * cur_norm)
        {
          converged = true;
          break;
        }
    }
  for (auto &e : ev)
    cudaEventDestroy(e);
  if (iterations)
    *iterations = step;
  if (last_update_norm)
    *last_update_norm = upd_cell_norm;
  if (rc)
    return rc;
  return converged ? DDHDG_OK : DDHDG_NOT_CONVERGED;
}

int
ddhdg_last_timings(const ddhdg_ctx *c, double *a, double *b, double *d, int *steps)
{
  if (!c)
    return fail(DDHDG_BAD_ARG, "null argument");
  if (a)
    *a = c->t_condense;
  if (b)
    *b = c->t_solve;
  if (d)
    *d = c->t_recon;
  if (steps)
    *steps = c->t_steps;
  return DDHDG_OK;
}

int
ddhdg_project_cell(ddhdg_ctx *c, const double *vals_cell, const double *vals_face, int comp,
                   double *cell_state, ddhdg_stream_t stream)
{
  if (!c || !vals_cell || !vals_face || !cell_state || comp < 0 || comp > 2)
    return fail(DDHDG_BAD_ARG, "bad argument");
  if (c->nb > 64 || c->nqf > 16)
    return fail(DDHDG_BAD_ARG, "projection supports (k+1)^d <= 64");
  project_cell_kernel<<<grid_for(c, c->ncells, 128), 128, 0, (cudaStream_t)stream>>>(
    c->ncells, c->dim, c->nb, c->nqc, c->nqf, c->F, c->tables.p, c->to, vals_cell, vals_face,
    comp, cell_state, 0, 0., 0., 0., 0., 0., 0.);
  CK(cudaGetLastError());
  return DDHDG_OK;
}

int
ddhdg_project_trace(ddhdg_ctx *c, const double *vals_face, int comp, double *trace_state,
                    ddhdg_stream_t stream)
{
  if (!c || !vals_face || !trace_state || comp < 0 || comp > 2)
    return fail(DDHDG_BAD_ARG, "bad argument");
  project_trace_kernel<<<grid_for(c, c->nfaces, 128), 128, 0, (cudaStream_t)stream>>>(
    c->nfaces, c->dim, c->nb, c->nf, c->nqf, c->F, c->tables.p, c->to, vals_face, comp,
    trace_state, 0, nullptr, nullptr, nullptr);
  CK(cudaGetLastError());
  return DDHDG_OK;
}

int
ddhdg_project_density(ddhdg_ctx *c, int comp, double qf, double *cell_state,
                      double *trace_state, ddhdg_stream_t stream)
{
  if (!c || !cell_state || !trace_state || (comp != 1 && comp != 2))
    return fail(DDHDG_BAD_ARG, "bad argument");
  if (c->nb > 64 || c->nqf > 16)
    return fail(DDHDG_BAD_ARG, "projection supports (k+1)^d <= 64");
  const auto  &d     = c->desc;
  const double nband = (comp == 1) ? d.nc : d.nv;
  const double eband = ((comp == 1) ? d.ec_eV : d.ev_eV) * EV_;
  project_cell_kernel<<<grid_for(c, c->ncells, 128), 128, 0, (cudaStream_t)stream>>>(
    c->ncells, c->dim, c->nb, c->nqc, c->nqf, c->F, c->tables.p, c->to, nullptr, nullptr, comp,
    cell_state, 1, qf, d.temperature, d.V_rescale, d.n_rescale, nband, eband);
  project_trace_kernel<<<grid_for(c, c->nfaces, 128), 128, 0, (cudaStream_t)stream>>>(
    c->nfaces, c->dim, c->nb, c->nf, c->nqf, c->F, c->tables.p, c->to, nullptr, comp,
    trace_state, 1, cell_state, c->d_face_cells.p, c->d_face_local.p);
  CK(cudaGetLastError());
  return DDHDG_OK;
}

} // extern "C"

// ---------------------------------------------------------------------------
// ddhdg_assemble_condense_noalloc: the condense launch of
// ddhdg_assemble_condense with its scratch (the per-cell Y cache and, for
// cells whose right-hand-side block does not fit in shared memory, that
// block) in a fixed static device array instead of context-owned buffers,
// so that the call allocates no device memory.

static __device__ __align__(256) double
  ddhdg_noalloc_scratch[DDHDG_NOALLOC_SCRATCH_BYTES / sizeof(double)];

namespace
{
  constexpr int NoAllocMaxDevices = 64;
  std::mutex    noalloc_mutex;
  double       *noalloc_ptr[NoAllocMaxDevices] = {};

  // Device address of the static scratch on the current device, looked up
  // once per device (the first call on a device must come before any stream
  // capture begins).
  int
  noalloc_scratch(double **out)
  {
    int dev = 0;
    CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= NoAllocMaxDevices)
      return fail(DDHDG_BAD_ARG, "device ordinal beyond the no-allocation scratch table");
    std::lock_guard<std::mutex> lock(noalloc_mutex);
    if (!noalloc_ptr[dev])
      {
        void             *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, ddhdg_noalloc_scratch);
        if (e != cudaSuccess || !p)
          {
            cudaGetLastError();
            return fail(DDHDG_CUDA_ERROR, std::string("cudaGetSymbolAddress of the static scratch: ") +
                                            cudaGetErrorString(e));
          }
        noalloc_ptr[dev] = static_cast<double *>(p);
      }
    *out = noalloc_ptr[dev];
    return DDHDG_OK;
  }
} // namespace

extern "C" {

int
ddhdg_assemble_condense_noalloc(ddhdg_ctx *c, const double *cell_state,
                                const double *trace_state, int thermo, double *tt,
                                double *rhs, int32_t *dflag, double *dval,
                                ddhdg_stream_t stream)
{
  if (!c || !cell_state || !trace_state || !tt || !rhs || !dflag || !dval)
    return fail(DDHDG_BAD_ARG, "null argument");
  thermo  = thermo ? 1 : 0;
  Mode &m = c->mode[thermo];
  if (!m.built)
    set_mode_comps(c, thermo); // host bookkeeping only; no trace sparsity needed here
  CondenseKernel cf;
  ReconstructFn rf;
  // the same kernel as ddhdg_assemble_condense: the FP32-Jacobian variant on
  // a mixed-precision context
  const bool mixed = c->desc.precision == 1;
  if (!kernels_for(c->dim, c->k, cf, rf, mixed))
    return fail(DDHDG_BAD_ARG, "unsupported dim/degree");
  int     r;
  KParams P     = make_params(c, thermo);
  P.cell_state  = cell_state;
  P.trace_state = trace_state;
  P.tt          = tt;
  P.rhs         = rhs;
  P.dflag       = dflag;
  P.dval        = dval;
  const int64_t Ns = (int64_t)m.ncomp * c->nb;
  int           threads;
  size_t        smem;
  int64_t       units;
  bool          r_global = false;
  if (3 * c->nb <= 32)
    {
      const Ws3Off w   = ws3_layout(c->dim, c->nb, c->nf, m.ncomp, m.ncol, mixed ? 4 : 8);
      const size_t per = (size_t)w.total * sizeof(double);
      int          wpb = (int)std::min<size_t>(Condense3MaxWPB, (mixed ? 110 : 220) * 1024 / per);
      if (wpb < 1)
        return fail(DDHDG_BAD_ARG, "the per-cell workspace does not fit in shared memory");
      P.wpb   = wpb;
      P.stage = 0;
      threads = wpb * 32;
      smem    = (size_t)wpb * per;
      units   = (c->ncells + wpb - 1) / wpb;
    }
  else
    {
      int stage;
      if ((r = launch_shape(c, m, stage, r_global, smem)))
        return r;
      P.wpb   = 1;
      P.stage = stage;
      threads = CondenseTPB;
      units   = c->ncells;
    }
  CK(allow_full_dynamic_smem(cf.fn));
  int per_sm = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, cf.fn, threads, smem));
  if (per_sm < 1)
    return fail(DDHDG_BAD_ARG, "condense kernel does not fit on an SM");
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(units, (int64_t)per_sm * c->sm_count));

  // scratch: Y cache [ncells][Ns][ycols], then (256-byte aligned) one R block
  // [Ns][ncol] per CTA when R lives outside shared memory
  const size_t ycache_n = (size_t)c->ncells * Ns * m.ycols;
  const size_t r_off    = (ycache_n + 31) & ~(size_t)31;
  const size_t need_n   = r_global ? r_off + (size_t)grid * Ns * m.ncol : ycache_n;
  if (need_n * sizeof(double) > DDHDG_NOALLOC_SCRATCH_BYTES)
    return fail(DDHDG_BAD_ARG,
                "this problem needs " + std::to_string(need_n * sizeof(double)) +
                  " bytes of condensation scratch; ddhdg_assemble_condense_noalloc holds at most " +
                  std::to_string((size_t)DDHDG_NOALLOC_SCRATCH_BYTES) +
                  " bytes (use ddhdg_assemble_condense)");
  double *scratch = nullptr;
  if ((r = noalloc_scratch(&scratch)))
    return r;
  P.ycache   = scratch;
  P.rscratch = r_global ? scratch + r_off : nullptr;

  // the status word must start at zero (a singular local system sets it)
  CK(cudaMemsetAsync(c->status.p, 0, sizeof(int), (cudaStream_t)stream));
  cf.launch(c->Tu, P, grid, threads, smem, (cudaStream_t)stream);
  CK(cudaGetLastError());
  return DDHDG_OK;
}

} // extern "C"

// ---------------------------------------------------------------------------
// The plain path: the reference's per-cell algorithm as written (full local
// system, LU of cc, Schur complement), and the per-cell probe.

namespace
{
  struct PlainKernel
  {
    const void *fn_smem = nullptr, *fn_glob = nullptr;
    void (*launch)(bool, const KParams &, const PlainArgs &, int, size_t, cudaStream_t) = nullptr;
  };

  template <int D, int K>
  void
  launch_plain(bool glob, const KParams &P, const PlainArgs &A, int grid, size_t smem, cudaStream_t s)
  {
    if (glob)
      plain_kernel<D, K, true><<<grid, PlainTPB, 0, s>>>(P, A);
    else
      plain_kernel<D, K, false><<<grid, PlainTPB, smem, s>>>(P, A);
  }

  template <int D, int K>
  void
  pick_plain(PlainKernel &pk)
  {
    pk.fn_smem = reinterpret_cast<const void *>(plain_kernel<D, K, false>);
    pk.fn_glob = reinterpret_cast<const void *>(plain_kernel<D, K, true>);
    pk.launch  = launch_plain<D, K>;
  }

  bool
  plain_for(int dim, int k, PlainKernel &pk)
  {
    switch (dim * 10 + k)
      {
        case 11: pick_plain<1, 1>(pk); return true;
        case 12: pick_plain<1, 2>(pk); return true;
        case 13: pick_plain<1, 3>(pk); return true;
        case 21: pick_plain<2, 1>(pk); return true;
        case 22: pick_plain<2, 2>(pk); return true;
        case 23: pick_plain<2, 3>(pk); return true;
        case 31: pick_plain<3, 1>(pk); return true;
        case 32: pick_plain<3, 2>(pk); return true;
        default: return false;
      }
  }

  // one launch of the plain kernel over `units` cells (or listed cells)
  int
  plain_run(ddhdg_ctx *c, int thermo, KParams &P, PlainArgs &A, int64_t units, cudaStream_t s)
  {
    PlainKernel pk;
    if (!plain_for(c->dim, c->k, pk))
      return fail(DDHDG_BAD_ARG, "unsupported dim/degree");
    Mode          &m    = c->mode[thermo];
    const PlainOff wo   = plain_layout(c->dim, c->nb, c->nf, m.ncomp, A.mode);
    const size_t   ws_b = (size_t)wo.total * sizeof(double);
    const bool     glob = ws_b > 220 * 1024;
    const void    *fn   = glob ? pk.fn_glob : pk.fn_smem;
    const size_t   smem = glob ? 0 : ws_b;
    if (!glob)
      CK(allow_full_dynamic_smem(fn));
    int per_sm = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, PlainTPB, smem));
    if (per_sm < 1)
      return fail(DDHDG_BAD_ARG, "plain kernel does not fit on an SM");
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(units, (int64_t)per_sm * c->sm_count));
    int       r;
    if (A.mode != PlainReconstruct)
      {
        if ((r = c->plain_tc.alloc((size_t)grid * wo.Nt * wo.Nc)))
          return r;
        A.tcscratch = c->plain_tc.p;
      }
    if (glob)
      {
        A.wstride = ((int64_t)wo.total + 31) & ~(int64_t)31;
        if ((r = c->plain_ws.alloc((size_t)grid * A.wstride)))
          return r;
        A.wscratch = c->plain_ws.p;
      }
    pk.launch(glob, P, A, grid, smem, s);
    CK(cudaGetLastError());
    return DDHDG_OK;
  }

  int
  plain_prepare(ddhdg_ctx *c, int thermo)
  {
    Mode &m = c->mode[thermo];
    if (!m.built)
      set_mode_comps(c, thermo); // host bookkeeping only; no trace sparsity needed here
    return DDHDG_OK;
  }
} // namespace

namespace
{
  struct SampleArgs
  {
    int     dim, k, nb, n[3];
    double  origin[3], h[3], gl[4];
    int     what; // 0 V, 1 n, 2 p (physical units); 3 phi_n, 4 phi_p (volts)
    double  V_rescale, n_rescale, T, ec, ev, nc, nv;
    int64_t npoints;
  };

  // get_solution_on_a_point (src/np_solver.cpp:1637-1700) for a batch of
  // points: the cell holding each point (on an interior face the cell above
  // it, outside the mesh the nearest boundary cell), the tensor-product
  // Lagrange basis on the Gauss-Lobatto support points there, and the scalar
  // of V, n or p in physical units, or a quasi Fermi potential from n or p
  // and V (compute_quasi_fermi_potential, include/solver.h:343-376).
  __global__ void
  sample_points_kernel(const SampleArgs A, const double *__restrict__ cell_state,
                       const double *__restrict__ pts, double *__restrict__ out)
  {
    const int NCA = 3 * (A.dim + 1) * A.nb;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < A.npoints;
         i += (int64_t)gridDim.x * blockDim.x)
      {
        int64_t cell = 0, stride = 1;
        double  lag[3][4];
        for (int a = 0; a < A.dim; ++a)
          {
            const double rel = (pts[i * 3 + a] - A.origin[a]) / A.h[a];
            int          ci  = (int)floor(rel);
            ci               = ci < 0 ? 0 : (ci > A.n[a] - 1 ? A.n[a] - 1 : ci);
            const double x   = rel - ci;
            for (int m = 0; m <= A.k; ++m)
              {
                double v = 1.;
                for (int j = 0; j <= A.k; ++j)
                  if (j != m)
                    v *= (x - A.gl[j]) / (A.gl[m] - A.gl[j]);
                lag[a][m] = v;
              }
            cell += ci * stride;
            stride *= A.n[a];
          }
        auto scalar = [&](int comp) {
          const double *cf = cell_state + cell * NCA + (comp * (A.dim + 1) + A.dim) * A.nb;
          double        s  = 0.;
          for (int b = 0; b < A.nb; ++b)
            {
              double phi = 1.;
              int    d   = b;
              for (int a = 0; a < A.dim; ++a)
                {
                  phi *= lag[a][d % (A.k + 1)];
                  d /= (A.k + 1);
                }
              s += phi * cf[b];
            }
          return s;
        };
        double r;
        if (A.what <= 2)
          r = scalar(A.what) * (A.what == 0 ? A.V_rescale : A.n_rescale);
        else
          {
            const double V   = scalar(0) * A.V_rescale;
            const double U_T = A.T * (KB_ / Q_);
            if (A.what == 3)
              r = V - A.ec / Q_ - U_T * log(scalar(1) * A.n_rescale / A.nc);
            else
              r = V - A.ev / Q_ + U_T * log(scalar(2) * A.n_rescale / A.nv);
          }
        out[i] = r;
      }
  }
} // namespace

extern "C" {

int
ddhdg_sample_points(ddhdg_ctx *c, const double *cell_state, int64_t npoints, const double *points,
                    int what, double *out, ddhdg_stream_t stream)
{
  if (!c || !cell_state || (npoints > 0 && (!points || !out)))
    return fail(DDHDG_BAD_ARG, "null argument");
  if (npoints < 0 || what < 0 || what > 4)
    return fail(DDHDG_BAD_ARG, "what must be 0 (V), 1 (n), 2 (p), 3 (phi_n) or 4 (phi_p)");
  if (npoints == 0)
    return DDHDG_OK;
  SampleArgs A{};
  A.dim = c->dim;
  A.k   = c->k;
  A.nb  = c->nb;
  for (int a = 0; a < 3; ++a)
    {
      A.n[a]      = (a < c->dim) ? c->desc.n[a] : 1;
      A.origin[a] = c->desc.origin[a];
      A.h[a]      = (a < c->dim) ? c->desc.h[a] : 1.;
    }
  for (int m = 0; m <= c->k && m < 4; ++m)
    A.gl[m] = c->T.gl[m];
  A.what      = what;
  A.V_rescale = c->desc.V_rescale;
  A.n_rescale = c->desc.n_rescale;
  A.T         = c->desc.temperature;
  A.ec        = c->desc.ec_eV * EV_;
  A.ev        = c->desc.ev_eV * EV_;
  A.nc        = c->desc.nc;
  A.nv        = c->desc.nv;
  A.npoints   = npoints;
  sample_points_kernel<<<grid_for(c, npoints, 256), 256, 0, (cudaStream_t)stream>>>(A, cell_state, points,
                                                                                   out);
  CK(cudaGetLastError());
  return DDHDG_OK;
}

int
ddhdg_local_cell_system(ddhdg_ctx *c, const double *cell_state, const double *trace_state,
                        int thermo, int64_t ncells, const int64_t *cells, int64_t first_cell,
                        double *cc, double *ct, double *tc, double *tt, double *cv, double *tv,
                        ddhdg_stream_t stream)
{
  if (!c || !cell_state || !trace_state)
    return fail(DDHDG_BAD_ARG, "null argument");
  if (ncells < 0 || (!cells && (first_cell < 0 || first_cell + ncells > c->ncells)))
    return fail(DDHDG_BAD_ARG, "cell range outside the mesh");
  if (ncells == 0)
    return DDHDG_OK;
  thermo = thermo ? 1 : 0;
  plain_prepare(c, thermo);
  KParams P     = make_params(c, thermo);
  P.cell_state  = cell_state;
  P.trace_state = trace_state;
  P.cell0       = first_cell;
  PlainArgs A{};
  A.mode  = PlainProbe;
  A.nlist = ncells;
  A.cells = cells;
  A.cc    = cc;
  A.ct    = ct;
  A.tc    = tc;
  A.tt    = tt;
  A.c     = cv;
  A.t     = tv;
  return plain_run(c, thermo, P, A, ncells, (cudaStream_t)stream);
}

int
ddhdg_assemble_condense_plain(ddhdg_ctx *c, const double *cell_state, const double *trace_state,
                              int thermo, double *tt, double *rhs, int32_t *dflag, double *dval,
                              ddhdg_stream_t stream)
{
  if (!c || !cell_state || !trace_state || !tt || !rhs || !dflag || !dval)
    return fail(DDHDG_BAD_ARG, "null argument");
  thermo = thermo ? 1 : 0;
  plain_prepare(c, thermo);
  KParams P     = make_params(c, thermo);
  P.cell_state  = cell_state;
  P.trace_state = trace_state;
  P.tt          = tt;
  P.rhs         = rhs;
  P.dflag       = dflag;
  P.dval        = dval;
  PlainArgs A{};
  A.mode = PlainCondense;
  return plain_run(c, thermo, P, A, c->ncells, (cudaStream_t)stream);
}

int
ddhdg_reconstruct_plain(ddhdg_ctx *c, const double *cell_state, const double *trace_state,
                        const double *update_trace, double *update_cell, int thermo,
                        ddhdg_stream_t stream)
{
  if (!c || !cell_state || !trace_state || !update_trace || !update_cell)
    return fail(DDHDG_BAD_ARG, "null argument");
  thermo = thermo ? 1 : 0;
  plain_prepare(c, thermo);
  KParams P     = make_params(c, thermo);
  P.cell_state  = cell_state;
  P.trace_state = trace_state;
  PlainArgs A{};
  A.mode         = PlainReconstruct;
  A.update_trace = update_trace;
  A.update_cell  = update_cell;
  return plain_run(c, thermo, P, A, c->ncells, (cudaStream_t)stream);
}

} // extern "C"

// ---------------------------------------------------------------------------
// Batched condensation / reconstruction over many contexts (devices of
// different mesh sizes and degrees, one dimension): one persistent launch
// each, consuming a work list of tiles; tile shapes from an autotuner.

struct ddhdg_batch
{
  int                      dim = 0, n = 0, thermo = 0;
  std::vector<ddhdg_ctx *> ctx;
  std::vector<BatchJob>    jobs;
  std::vector<int64_t>     ncells, ycache_off;
  std::vector<double>      cost_per_cell; // per job, for the heaviest-first order
  DevBuf<unsigned char>    d_jobs, d_tiles_c, d_tiles_r;
  DevBuf<double>           ycache, rscratch;
  DevBuf<int>              counter; // [0]: condense, [1]: reconstruct
  bool                     degrees[4]        = {false, false, false, false};
  int                      cells_per_tile[4] = {0, 32, 32, 4};
  int                      ctas_per_sm       = 8; // at most; the kernel's occupancy limit applies
  int                      occ_c             = 0; // CTAs per SM the condense kernel allows
  int                      rcells_per_tile   = 256;
  int                      ntiles_c = 0, ntiles_r = 0, grid_c = 0, grid_r = 0;
  size_t                   smem_c = 0, smem_r = 0;
  bool                     any_r_global         = false;
  int                      prec                 = BatchFP64; // the precisions of the jobs
  int                      max_rscratch_per_cta = 0;
  int                      sm_count             = 148;
  cudaStream_t             cap                  = nullptr;
  cudaGraphExec_t          g_c = nullptr, g_r = nullptr;
  // Newton steps: norm words and side streams
  static constexpr int     NS = 8;
  DevBuf<unsigned long long> norms;
  cudaStream_t             side[NS] = {};
  cudaEvent_t              ev_fork = nullptr, ev_join[NS] = {};
  // a step begun and not yet ended: its stream, its completion event and
  // the pinned host copies of its norms and statuses
  bool                     pending  = false;
  cudaStream_t             step_s   = nullptr;
  cudaEvent_t              ev_done  = nullptr;
  double                  *h_norms  = nullptr;
  int                     *h_status = nullptr;
  ~ddhdg_batch()
  {
    if (pending && ev_done)
      cudaEventSynchronize(ev_done);
    if (ev_done)
      cudaEventDestroy(ev_done);
    if (h_norms)
      cudaFreeHost(h_norms);
    if (h_status)
      cudaFreeHost(h_status);
    for (auto &st : side)
      if (st)
        cudaStreamDestroy(st);
    for (auto &e : ev_join)
      if (e)
        cudaEventDestroy(e);
    if (ev_fork)
      cudaEventDestroy(ev_fork);
    if (g_c)
      cudaGraphExecDestroy(g_c);
    if (g_r)
      cudaGraphExecDestroy(g_r);
    if (cap)
      cudaStreamDestroy(cap);
  }
};

namespace
{
  template <int D>
  const void *
  batch_condense_fn_d(int prec)
  {
    switch (prec)
      {
        case BatchFP64: return reinterpret_cast<const void *>(batch_condense_kernel<D, BatchFP64>);
        case BatchMixed: return reinterpret_cast<const void *>(batch_condense_kernel<D, BatchMixed>);
        default: return reinterpret_cast<const void *>(batch_condense_kernel<D, BatchBoth>);
      }
  }
  const void *
  batch_condense_fn(int dim, int prec)
  {
    switch (dim)
      {
        case 1: return batch_condense_fn_d<1>(prec);
        case 2: return batch_condense_fn_d<2>(prec);
        default: return batch_condense_fn_d<3>(prec);
      }
  }
  const void *
  batch_reconstruct_fn(int dim)
  {
    switch (dim)
      {
        case 1: return reinterpret_cast<const void *>(batch_reconstruct_kernel<1>);
        case 2: return reinterpret_cast<const void *>(batch_reconstruct_kernel<2>);
        default: return reinterpret_cast<const void *>(batch_reconstruct_kernel<3>);
      }
  }

  // the unit-cell constant tables of every warp-per-cell degree of DIM
  template <int D>
  void
  fill_batch_tabs(BatchTabs<D> &C)
  {
    const double unit[3] = {1., 1., 1.};
    if constexpr (batch_warp<D, 1>)
      fill_ctab(build_tables(D, 1, unit), C.t1);
    if constexpr (batch_warp<D, 2>)
      fill_ctab(build_tables(D, 2, unit), C.t2);
    if constexpr (batch_warp<D, 3>)
      fill_ctab(build_tables(D, 3, unit), C.t3);
  }

  // work lists and launch shapes for the current tile sizes
  int
  batch_plan(ddhdg_batch *b)
  {
    if (b->g_c)
      {
        cudaGraphExecDestroy(b->g_c);
        b->g_c = nullptr;
      }
    if (b->g_r)
      {
        cudaGraphExecDestroy(b->g_r);
        b->g_r = nullptr;
      }
    const void *fc = batch_condense_fn(b->dim, b->prec), *fr = batch_reconstruct_fn(b->dim);
    CK(allow_full_dynamic_smem(fc));
    CK(allow_full_dynamic_smem(fr));
    int per_sm_r = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_r, fr, BatchRTPB, b->smem_r));
    if (per_sm_r < 1)
      return fail(DDHDG_BAD_ARG, "batched reconstruction kernel does not fit on an SM");
    // reconstruction tiles: at most rcells_per_tile cells, and small enough
    // that every CTA of a full grid gets about four
    int64_t rtile;
    {
      int64_t total = 0;
      for (int64_t nc : b->ncells)
        total += nc;
      const int64_t fill = total / ((int64_t)per_sm_r * b->sm_count * 4);
      rtile              = std::max<int64_t>(16, std::min<int64_t>(b->rcells_per_tile, fill));
    }
    std::vector<BatchTile> tc, tr;
    for (int j = 0; j < b->n; ++j)
      {
        const int     k  = b->jobs[j].k;
        const int64_t nc = b->ncells[j];
        const int64_t T  = std::max(1, b->cells_per_tile[k]);
        for (int64_t c0 = 0; c0 < nc; c0 += T)
          tc.push_back(BatchTile{j, 0, c0, std::min(nc, c0 + T)});
        for (int64_t c0 = 0; c0 < nc; c0 += rtile)
          tr.push_back(BatchTile{j, 0, c0, std::min<int64_t>(nc, c0 + rtile)});
      }
    // heaviest tiles first, so that the last tiles handed out are short
    auto cost = [b](const BatchTile &t) { return (double)(t.end - t.begin) * b->cost_per_cell[t.job]; };
    std::stable_sort(tc.begin(), tc.end(),
                     [&](const BatchTile &x, const BatchTile &y) { return cost(x) > cost(y); });
    int r;
    if ((r = b->d_tiles_c.upload(reinterpret_cast<const unsigned char *>(tc.data()), tc.size() * sizeof(BatchTile))))
      return r;
    if ((r = b->d_tiles_r.upload(reinterpret_cast<const unsigned char *>(tr.data()), tr.size() * sizeof(BatchTile))))
      return r;
    b->ntiles_c     = (int)tc.size();
    b->ntiles_r     = (int)tr.size();
    int per_sm = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fc, BatchTPB, b->smem_c));
    if (per_sm < 1)
      return fail(DDHDG_BAD_ARG, "batched condense kernel does not fit on an SM");
    b->occ_c  = per_sm;
    b->grid_c = std::max(1, std::min(b->ntiles_c, std::min(per_sm, b->ctas_per_sm) * b->sm_count));

    b->grid_r = std::max(1, std::min(b->ntiles_r, per_sm_r * b->sm_count));
    // R blocks outside shared memory (3D degree 2): one slice per CTA
    if (b->any_r_global)
      {
        if ((r = b->rscratch.alloc((size_t)b->grid_c * b->max_rscratch_per_cta)))
          return r;
        for (auto &J : b->jobs)
          if (J.P.rscratch)
            J.P.rscratch = b->rscratch.p;
        if ((r = b->d_jobs.upload(reinterpret_cast<const unsigned char *>(b->jobs.data()),
                                  b->jobs.size() * sizeof(BatchJob))))
          return r;
      }
    return DDHDG_OK;
  }

  template <int D>
  void
  batch_launch_condense_d(ddhdg_batch *b, const BatchJob *jobs, const BatchTile *tiles, cudaStream_t s)
  {
    static BatchTabs<D>   C; // filled once; the tables do not depend on the device
    static std::once_flag once;
    std::call_once(once, [] { fill_batch_tabs<D>(C); });
    if (b->prec == BatchFP64)
      batch_condense_kernel<D, BatchFP64><<<b->grid_c, BatchTPB, b->smem_c, s>>>(jobs, tiles, b->ntiles_c, b->counter.p, C);
    else if (b->prec == BatchMixed)
      batch_condense_kernel<D, BatchMixed><<<b->grid_c, BatchTPB, b->smem_c, s>>>(jobs, tiles, b->ntiles_c, b->counter.p, C);
    else
      batch_condense_kernel<D, BatchBoth><<<b->grid_c, BatchTPB, b->smem_c, s>>>(jobs, tiles, b->ntiles_c, b->counter.p, C);
  }

  int
  batch_launch_condense(ddhdg_batch *b, cudaStream_t s)
  {
    CK(cudaMemsetAsync(b->counter.p, 0, sizeof(int), s));
    const BatchJob  *jobs  = reinterpret_cast<const BatchJob *>(b->d_jobs.p);
    const BatchTile *tiles = reinterpret_cast<const BatchTile *>(b->d_tiles_c.p);
    switch (b->dim)
      {
        case 1: batch_launch_condense_d<1>(b, jobs, tiles, s); break;
        case 2: batch_launch_condense_d<2>(b, jobs, tiles, s); break;
        default: batch_launch_condense_d<3>(b, jobs, tiles, s); break;
      }
    CK(cudaGetLastError());
    return DDHDG_OK;
  }

  int
  batch_launch_reconstruct(ddhdg_batch *b, cudaStream_t s)
  {
    CK(cudaMemsetAsync(b->counter.p + 1, 0, sizeof(int), s));
    const BatchJob  *jobs  = reinterpret_cast<const BatchJob *>(b->d_jobs.p);
    const BatchTile *tiles = reinterpret_cast<const BatchTile *>(b->d_tiles_r.p);
    int             *cnt   = b->counter.p + 1;
    switch (b->dim)
      {
        case 1:
          batch_reconstruct_kernel<1><<<b->grid_r, BatchRTPB, b->smem_r, s>>>(jobs, tiles, b->ntiles_r, cnt);
          break;
        case 2:
          batch_reconstruct_kernel<2><<<b->grid_r, BatchRTPB, b->smem_r, s>>>(jobs, tiles, b->ntiles_r, cnt);
          break;
        default:
          batch_reconstruct_kernel<3><<<b->grid_r, BatchRTPB, b->smem_r, s>>>(jobs, tiles, b->ntiles_r, cnt);
          break;
      }
    CK(cudaGetLastError());
    return DDHDG_OK;
  }

  // replay of the launch from a CUDA graph captured on the first call (on
  // an internal stream, thread-local capture); eager launch if capture fails
  int
  batch_run(ddhdg_batch *b, cudaStream_t s, bool recon)
  {
    cudaGraphExec_t &ge = recon ? b->g_r : b->g_c;
    if (!ge)
      {
        if (!b->cap)
          CK(cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking));
        cudaGraph_t g = nullptr;
        if (cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal) == cudaSuccess)
          {
            const int         rr = recon ? batch_launch_reconstruct(b, b->cap) : batch_launch_condense(b, b->cap);
            const cudaError_t e  = cudaStreamEndCapture(b->cap, &g);
            if (rr == DDHDG_OK && e == cudaSuccess && g)
              {
                if (cudaGraphInstantiate(&ge, g, 0) != cudaSuccess)
                  ge = nullptr;
              }
            if (g)
              cudaGraphDestroy(g);
          }
        cudaGetLastError();
      }
    if (ge)
      {
        CK(cudaGraphLaunch(ge, s));
        return DDHDG_OK;
      }
    return recon ? batch_launch_reconstruct(b, s) : batch_launch_condense(b, s);
  }

  // best of `reps` eager launches of the batched condensation (after one
  // warm-up launch), by CUDA events on s
  int
  batch_time(ddhdg_batch *b, cudaStream_t s, int reps, float &ms)
  {
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    int   r    = batch_launch_condense(b, s);
    float best = 1e30f;
    for (int i = 0; i < reps && r == DDHDG_OK; ++i)
      {
        cudaEventRecord(e0, s);
        r = batch_launch_condense(b, s);
        cudaEventRecord(e1, s);
        if (cudaEventSynchronize(e1) != cudaSuccess)
          r = fail(DDHDG_CUDA_ERROR, "batched condense launch failed");
        float t = 0.f;
        cudaEventElapsedTime(&t, e0, e1);
        best = std::min(best, t);
      }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    ms = best;
    return r;
  }
} // namespace

extern "C" {

int
ddhdg_batch_create(const ddhdg_batch_item *items, int n, int thermo, ddhdg_batch **out)
{
  if (!items || n < 1 || !out)
    return fail(DDHDG_BAD_ARG, "null argument or empty batch");
  thermo = thermo ? 1 : 0;
  std::unique_ptr<ddhdg_batch> b(new ddhdg_batch);
  b->n      = n;
  b->thermo = thermo;
  b->dim    = items[0].ctx ? items[0].ctx->dim : 0;
  int64_t                    ytotal = 0;
  int                        r;
  for (int j = 0; j < n; ++j)
    {
      const ddhdg_batch_item &it = items[j];
      ddhdg_ctx              *c  = it.ctx;
      if (!c || !it.cell_state || !it.trace_state || !it.tt || !it.rhs || !it.dflag || !it.dval)
        return fail(DDHDG_BAD_ARG, "batch item " + std::to_string(j) + ": null argument");
      if (c->dim != b->dim)
        return fail(DDHDG_BAD_ARG, "batch items must share one dimension");
      Mode &m = c->mode[thermo];
      if (!m.built)
        set_mode_comps(c, thermo); // host bookkeeping only
      b->ctx.push_back(c);
      b->ncells.push_back(c->ncells);
      b->sm_count = c->sm_count;
      BatchJob J{};
      J.P             = make_params(c, thermo);
      J.P.cell0       = 0;
      J.P.ncells      = c->ncells;
      J.P.cell_state  = it.cell_state;
      J.P.trace_state = it.trace_state;
      J.P.tt          = it.tt;
      J.P.rhs         = it.rhs;
      J.P.dflag       = it.dflag;
      J.P.dval        = it.dval;
      J.dtrace        = it.update_trace;
      J.dcell         = it.update_cell;
      J.k             = c->k;
      J.mixed         = c->desc.precision == 1 ? 1 : 0; // only where 3 nb <= 32 (ctx_create)
      {
        const int jp = J.mixed ? BatchMixed : BatchFP64;
        b->prec      = (j == 0 || b->prec == jp) ? jp : BatchBoth;
      }
      const int Ns    = m.ncomp * c->nb;
      b->ycache_off.push_back(ytotal);
      ytotal += ((c->ncells * Ns * m.ycols) + 31) & ~(int64_t)31;
      b->degrees[c->k] = true;
      // Ns^3 (inverse) + Ns^2 (1 + Nt) (Y) + Nt^2 Ns (tt): heaviest-first order
      b->cost_per_cell.push_back((double)Ns * Ns * Ns + (double)Ns * Ns * (1 + m.Nt) +
                                 (double)m.Nt * m.Nt * Ns);
      if (3 * c->nb <= 32)
        {
          const Ws3Off w = ws3_layout(c->dim, c->nb, c->nf, m.ncomp, m.ncol, J.mixed ? 4 : 8);
          // the warps' workspaces and the staged face-flux table
          b->smem_c = std::max(b->smem_c, ((size_t)BatchWarp * w.total +
                                           (size_t)(c->F * c->nqf) * (c->F * c->nf)) * sizeof(double));
          J.P.wpb        = 1;
          J.P.stage      = 0;
        }
      else
        {
          // the tables are read through L1 (not staged); R stays in shared
          // memory if that keeps two CTAs on an SM, else if it fits at all,
          // else it moves to global memory (no choice changes the arithmetic)
          bool   found = false, r_global = false;
          size_t smem  = 0;
          for (size_t limit : {(size_t)110 * 1024, (size_t)220 * 1024})
            {
              for (int rg = 0; rg < 2 && !found; ++rg)
                {
                  const Ws2Off w = ws2_layout(c->dim, c->nb, c->nf, m.ncomp, m.ncol, rg != 0);
                  if ((size_t)w.total * sizeof(double) <= limit)
                    {
                      found    = true;
                      r_global = rg != 0;
                      smem     = (size_t)w.total * sizeof(double);
                    }
                }
              if (found)
                break;
            }
          if (!found)
            return fail(DDHDG_BAD_ARG, "the per-cell workspace does not fit in shared memory");
          J.P.wpb   = 1;
          J.P.stage = 0;
          b->smem_c = std::max(b->smem_c, smem);
          if (r_global)
            {
              b->any_r_global         = true;
              b->max_rscratch_per_cta = std::max(b->max_rscratch_per_cta, Ns * m.ncol);
              J.P.rscratch            = reinterpret_cast<double *>(1); // set by batch_plan
            }
        }
      // reconstruction workspace (reconstruct_cells with BatchRTPB / 32 warps)
      const size_t nPQ = (size_t)(c->to.minv - c->to.P);
      const int    wsz = (Ns + 2 * c->F * 3 * c->nf + c->nb + m.Nt + 1) & ~1;
      b->smem_r = std::max(b->smem_r,
                           (((nPQ + 1) & ~(size_t)1) + (size_t)(BatchRTPB / 32) * wsz) * sizeof(double));
      b->jobs.push_back(J);
    }
  if ((r = b->ycache.alloc((size_t)ytotal)))
    return r;
  for (int j = 0; j < n; ++j)
    b->jobs[j].P.ycache = b->ycache.p + b->ycache_off[j];
  if ((r = b->counter.alloc(2)))
    return r;
  if ((r = b->d_jobs.upload(reinterpret_cast<const unsigned char *>(b->jobs.data()),
                            b->jobs.size() * sizeof(BatchJob))))
    return r;
  if ((r = batch_plan(b.get())))
    return r;
  *out = b.release();
  return DDHDG_OK;
}

int
ddhdg_batch_destroy(ddhdg_batch *b)
{
  delete b;
  return DDHDG_OK;
}

int
ddhdg_batch_condense(ddhdg_batch *b, ddhdg_stream_t stream)
{
  if (!b)
    return fail(DDHDG_BAD_ARG, "null argument");
  return batch_run(b, (cudaStream_t)stream, false);
}

int
ddhdg_batch_reconstruct(ddhdg_batch *b, ddhdg_stream_t stream)
{
  if (!b)
    return fail(DDHDG_BAD_ARG, "null argument");
  for (const auto &J : b->jobs)
    if (!J.dtrace || !J.dcell)
      return fail(DDHDG_BAD_ARG, "a batch item has no update_trace / update_cell");
  return batch_run(b, (cudaStream_t)stream, true);
}

int
ddhdg_batch_newton_step_begin(ddhdg_batch *b, const double *alpha, ddhdg_stream_t stream)
{
  if (!b || !alpha)
    return fail(DDHDG_BAD_ARG, "null argument");
  if (b->pending)
    return fail(DDHDG_BAD_ARG, "the batch has a step that has not ended");
  for (const auto &J : b->jobs)
    if (!J.dtrace || !J.dcell)
      return fail(DDHDG_BAD_ARG, "a batch item has no update_trace / update_cell");
  cudaStream_t s = (cudaStream_t)stream;
  const int    n = b->n;
  int          r;
  if (!b->ev_fork)
    {
      // each item's restricted trace solution lives in its context (the
      // same buffer whatever batch the context is in, so that the context's
      // trace-solve graph stays valid across batches)
      for (int i = 0; i < n; ++i)
        {
          ddhdg_ctx *c = b->ctx[i];
          Mode      &m = c->mode[b->thermo];
          if (!m.built && (r = build_mode(c, b->thermo)))
            return r;
          if ((r = m.x.alloc(m.ndofs)))
            return r;
        }
      if ((r = b->norms.alloc((size_t)4 * n)))
        return r;
      for (int k = 0; k < ddhdg_batch::NS; ++k)
        {
          CK(cudaStreamCreateWithFlags(&b->side[k], cudaStreamNonBlocking));
          CK(cudaEventCreateWithFlags(&b->ev_join[k], cudaEventDisableTiming));
        }
      CK(cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming));
      CK(cudaEventCreateWithFlags(&b->ev_done, cudaEventDisableTiming));
      CK(cudaMallocHost(reinterpret_cast<void **>(&b->h_norms), (size_t)4 * n * sizeof(double)));
      CK(cudaMallocHost(reinterpret_cast<void **>(&b->h_status), (size_t)n * sizeof(int)));
    }
  for (int i = 0; i < n; ++i)
    CK(cudaMemsetAsync(b->ctx[i]->status.p, 0, sizeof(int), s));
  // 1) one launch: assembly + condensation of every item
  if ((r = batch_run(b, s, false)))
    return r;
  // 2) every item's trace solve, on side streams so that they overlap
  CK(cudaEventRecord(b->ev_fork, s));
  const int used = std::min(n, ddhdg_batch::NS);
  for (int k = 0; k < used; ++k)
    CK(cudaStreamWaitEvent(b->side[k], b->ev_fork, 0));
  for (int i = 0; i < n; ++i)
    {
      ddhdg_ctx     *c  = b->ctx[i];
      Mode          &m  = c->mode[b->thermo];
      const BatchJob &J = b->jobs[i];
      cudaStream_t   ss = b->side[i % ddhdg_batch::NS];
      NDSolver      *nd = nullptr;
      if ((r = nd_solver(c, m, nd)))
        return r;
      std::string err;
      if ((r = nd->solve(J.P.tt, J.P.rhs, J.P.dflag, J.P.dval, m.Nt, m.x.p, ss, c->sm_count, err, false)))
        return fail(r, err);
      const int64_t ntr = c->nfaces * 3 * c->nf;
      expand_kernel<<<grid_for(c, ntr, 256), 256, 0, ss>>>(c->nfaces, c->nf, m.ncomp, m.comps[0], m.comps[1],
                                                           m.comps[2], m.x.p, const_cast<double *>(J.dtrace));
    }
  for (int k = 0; k < used; ++k)
    {
      CK(cudaEventRecord(b->ev_join[k], b->side[k]));
      CK(cudaStreamWaitEvent(s, b->ev_join[k], 0));
    }
  // 3) one launch: reconstruction of every item
  if ((r = batch_run(b, s, true)))
    return r;
  // 4) norms before the update, then state += alpha (dcell, dtrace)
  CK(cudaMemsetAsync(b->norms.p, 0, (size_t)4 * n * sizeof(unsigned long long), s));
  for (int i = 0; i < n; ++i)
    {
      ddhdg_ctx     *c   = b->ctx[i];
      const BatchJob &J  = b->jobs[i];
      const int64_t  ncd = c->ncells * 3 * (c->dim + 1) * c->nb;
      const int64_t  ntr = c->nfaces * 3 * c->nf;
      absmax_kernel<<<grid_for(c, ncd, 256), 256, 0, s>>>(J.dcell, ncd, J.dtrace, ntr, J.P.cell_state, ncd,
                                                          J.P.trace_state, ntr, b->norms.p + 4 * i);
      axpy2_kernel<<<grid_for(c, ncd + ntr, 256), 256, 0, s>>>(ntr, const_cast<double *>(J.P.trace_state),
                                                               J.dtrace, ncd,
                                                               const_cast<double *>(J.P.cell_state), J.dcell,
                                                               alpha[i]);
    }
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(b->h_norms, b->norms.p, (size_t)4 * n * sizeof(double), cudaMemcpyDeviceToHost, s));
  for (int i = 0; i < n; ++i)
    CK(cudaMemcpyAsync(b->h_status + i, b->ctx[i]->status.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  CK(cudaEventRecord(b->ev_done, s));
  b->step_s  = s;
  b->pending = true;
  return DDHDG_OK;
}

int
ddhdg_batch_newton_step_end(ddhdg_batch *b, int wait, double *norms_host, int *status_host, int *done)
{
  if (!b || !norms_host || !done)
    return fail(DDHDG_BAD_ARG, "null argument");
  *done = 0;
  if (!b->pending)
    return fail(DDHDG_BAD_ARG, "the batch has no step in flight");
  if (!wait)
    {
      const cudaError_t q = cudaEventQuery(b->ev_done);
      if (q == cudaErrorNotReady)
        return DDHDG_OK;
      if (q != cudaSuccess)
        return fail(DDHDG_CUDA_ERROR, cudaGetErrorString(q));
    }
  else
    CK(cudaEventSynchronize(b->ev_done));
  b->pending = false;
  *done      = 1;
  const int n = b->n;
  std::memcpy(norms_host, b->h_norms, (size_t)4 * n * sizeof(double));
  // singular fronts of the trace solves (their pivot status, read now)
  int worst = DDHDG_OK;
  for (int i = 0; i < n; ++i)
    {
      ddhdg_ctx  *c  = b->ctx[i];
      NDSolver   *nd = nullptr;
      std::string err;
      int         st = b->h_status[i];
      if (nd_solver(c, c->mode[b->thermo], nd) == DDHDG_OK && nd->check_info(b->step_s, err) != DDHDG_OK)
        st = DDHDG_SOLVER_ERROR;
      if (status_host)
        status_host[i] = st;
      if (st && !worst)
        worst = st;
    }
  if (worst)
    return fail(worst, "a batch item had a singular local system or trace front (see the item statuses)");
  return DDHDG_OK;
}

int
ddhdg_batch_newton_step(ddhdg_batch *b, const double *alpha, double *norms_host, int *status_host,
                        ddhdg_stream_t stream)
{
  if (!b || !alpha || !norms_host)
    return fail(DDHDG_BAD_ARG, "null argument");
  int r, done = 0;
  if ((r = ddhdg_batch_newton_step_begin(b, alpha, stream)))
    return r;
  return ddhdg_batch_newton_step_end(b, 1, norms_host, status_host, &done);
}

int
ddhdg_batch_set_shape(ddhdg_batch *b, const int *cells_per_tile, int ctas_per_sm)
{
  if (!b || !cells_per_tile || ctas_per_sm < 1)
    return fail(DDHDG_BAD_ARG, "null argument or no CTA per SM");
  for (int k = 1; k <= 3; ++k)
    if (cells_per_tile[k - 1] < 1)
      return fail(DDHDG_BAD_ARG, "cells per tile must be positive");
  for (int k = 1; k <= 3; ++k)
    b->cells_per_tile[k] = cells_per_tile[k - 1];
  b->ctas_per_sm = ctas_per_sm;
  return batch_plan(b);
}

int
ddhdg_batch_get_shape(const ddhdg_batch *b, int *cells_per_tile, int *ctas_per_sm, int *grid,
                      int *ntiles)
{
  if (!b)
    return fail(DDHDG_BAD_ARG, "null argument");
  for (int k = 1; k <= 3 && cells_per_tile; ++k)
    cells_per_tile[k - 1] = b->cells_per_tile[k];
  if (ctas_per_sm)
    *ctas_per_sm = b->ctas_per_sm;
  if (grid)
    *grid = b->grid_c;
  if (ntiles)
    *ntiles = b->ntiles_c;
  return DDHDG_OK;
}

int
ddhdg_batch_autotune(ddhdg_batch *b, int reps, float *best_ms, ddhdg_stream_t stream)
{
  if (!b)
    return fail(DDHDG_BAD_ARG, "null argument");
  reps           = std::max(1, reps);
  cudaStream_t s = (cudaStream_t)stream;
  int          r;
  float        best = 0.f;
  if ((r = batch_time(b, s, reps, best)))
    return r;
  // coordinate search: the tile size of each degree present (heaviest
  // degree first), then the CTAs per SM
  const int warp_cand[] = {4, 8, 16, 32, 64, 128, 256};
  const int cta_cand[]  = {1, 2, 4, 8, 16, 32};
  for (int k = 3; k >= 1; --k)
    {
      if (!b->degrees[k])
        continue;
      int nbk = 1;
      for (int a = 0; a < b->dim; ++a)
        nbk *= k + 1;
      const bool cta  = 3 * nbk > 32;
      const int *cand = cta ? cta_cand : warp_cand;
      const int  nc   = cta ? 6 : 7;
      int        keep = b->cells_per_tile[k];
      for (int i = 0; i < nc; ++i)
        {
          if (cand[i] == keep)
            continue;
          b->cells_per_tile[k] = cand[i];
          float t              = 0.f;
          if ((r = batch_plan(b)) || (r = batch_time(b, s, reps, t)))
            return r;
          if (t < best)
            {
              best = t;
              keep = cand[i];
            }
          b->cells_per_tile[k] = keep;
        }
    }
  // CTAs per SM: 1 up to what the kernel's registers and the batch's
  // shared memory allow (at most 8)
  b->ctas_per_sm = std::min(b->ctas_per_sm, b->occ_c);
  for (int cps = 1; cps <= std::min(8, b->occ_c); ++cps)
    {
      if (cps == b->ctas_per_sm)
        continue;
      const int prev = b->ctas_per_sm;
      b->ctas_per_sm = cps;
      float t        = 0.f;
      if ((r = batch_plan(b)) || (r = batch_time(b, s, reps, t)))
        return r;
      if (t < best)
        best = t;
      else
        b->ctas_per_sm = prev;
    }
  if ((r = batch_plan(b)))
    return r;
  if (best_ms)
    *best_ms = best;
  return DDHDG_OK;
}

} // extern "C"
