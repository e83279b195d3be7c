// Strided FFT passes with tensor-memory-accelerator (TMA) staging: the middle passes of the 3D schedule (forward
// or inverse along a strided axis) and the axis-0 pass with the fused dyadic Green multiply, complex64.
//
// A tile is the same 16-pencil tile as k_reg_pass's: C components x N samples x 16 consecutive pencils, stored in
// shared memory as [c][j][pencil] with 128-byte rows.  That is exactly the dense box of a 5-D tensor map over the
// work buffer T [B][C][outer][N][inner] (innermost first: inner, N, outer, C, B; box 16 x N x 1 x C x 1), so one
// cp.async.bulk.tensor load brings a whole 48 KB tile (C = 3, N = 128) into shared memory and one bulk tensor store
// writes it back.  The threads never touch global memory: every radix stage runs shared -> registers -> shared
// (rstage with FROM_G = TO_G = false), and the Green stage of the axis-0 pass is green_fused_vector/_scalar.
//
// Each CTA is persistent over the tiles blockIdx.x, blockIdx.x + gridDim.x, ... and owns two tile buffers: while
// it transforms one tile, the load of its next tile is in flight in the other buffer and the store of its previous
// tile drains.  Buffer s is refilled (with the tile two steps ahead) only after the bulk store from it has finished
// reading shared memory (cp.async.bulk.wait_group.read).  Loads complete on one mbarrier per buffer; the waits are
// bounded (2^20 polls): on a timeout the tile is skipped, MMX_STATUS_TIMEOUT is raised in the right-hand side's
// state and the copy is drained (bounded again) before the buffer is re-armed.  The tensor map covers only this
// GPU's own work buffer; no load uses cluster multicast.
#pragma once
#include <cuda.h>

#include "mmx_reg.cuh"

namespace mmx_tma {

// shared-memory address of a generic pointer into shared memory
__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void load_tile(void* dst, const CUtensorMap* map, int c0, int c1, int c2, int c3, int c4,
                                          uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, "
      "%6}], [%7];" ::"r"(smem_u32(dst)),
      "l"((uint64_t)map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void store_tile(const CUtensorMap* map, int c0, int c1, int c2, int c3, int c4,
                                           const void* src) {
  asm volatile("cp.async.bulk.tensor.5d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3, %4, %5}], [%6];" ::"l"(
                   (uint64_t)map),
               "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(smem_u32(src))
               : "memory");
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}

// the bulk stores issued by this thread have finished reading shared memory
__device__ __forceinline__ void stores_read_done() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
// ... and have completed
__device__ __forceinline__ void stores_done() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
// order this thread's generic-proxy shared-memory accesses before later async-proxy (bulk copy) accesses
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

template <int C, int N> struct Layout {
  static constexpr int P = kRegP;
  static constexpr int TILE = C * N * P;  // words per tile buffer
  static constexpr unsigned TILE_BYTES = TILE * sizeof(float2);
  // two tile buffers (128-byte aligned) and the twiddle table
  static constexpr size_t bytes() { return (size_t)2 * TILE * sizeof(float2) + (size_t)N * sizeof(float2) + 128; }
};

}  // namespace mmx_tma

// OPS: OP_FWD, OP_INV, or OP_FWD | OP_G | OP_INV (axis-0 pass).  tiles_per_rhs = outer * inner / 16.
template <int C, int OPS, int N>
__global__ void __launch_bounds__(RegThreads<C, N>::value, 2)
    k_tma_pass(IterArgs<float> a, const __grid_constant__ CUtensorMap tmap, int tiles_per_rhs) {
  using namespace mmx_tma;
  using LY = Layout<C, N>;
  constexpr int P = kRegP;
  constexpr int THREADS = RegThreads<C, N>::value;
  extern __shared__ __align__(16) unsigned char mmx_smem_raw[];
  // 128-byte aligned tile buffers (the dynamic shared window is at least 16-byte aligned)
  float2* buf0 = reinterpret_cast<float2*>((reinterpret_cast<uintptr_t>(mmx_smem_raw) + 127) & ~uintptr_t(127));
  float2* smtw = buf0 + 2 * LY::TILE;
  __shared__ __align__(8) uint64_t bars[2];
  __shared__ int s_active[2];
  __shared__ float sk1[P], sk2[P], sk0[N];
  const int tid = threadIdx.x;
  const int64_t inner = a.inner;
  const int nrhs = a.nrhs;
  const int64_t ntiles = (int64_t)tiles_per_rhs * nrhs;
  const float2* twg = (const float2*)a.ax.tw;
  for (int t = tid; t < N; t += THREADS) smtw[t] = twg[t];
  if constexpr ((OPS & OP_G) != 0) {
    for (int t = tid; t < N; t += THREADS) sk0[t] = a.kv[0][t];
  }
  pdl_wait();  // T and the states are written by earlier passes
  pdl_trigger();

  // tile t -> tensor coordinates (pencil offset, 0, outer index, 0, rhs)
  auto coords = [&](int64_t t, int& c0, int& c2, int& c4) {
    const int b = (int)(t / tiles_per_rhs);
    const int64_t p0 = (t % tiles_per_rhs) * P;
    const int64_t o = p0 / inner;
    c0 = (int)(p0 - o * inner);
    c2 = (int)o;
    c4 = b;
  };
  auto issue = [&](int s, int64_t t) {  // thread 0 only
    int c0, c2, c4;
    coords(t, c0, c2, c4);
    const int active = a.st[c4].active;
    s_active[s] = active;
    if (!active) {  // complete this phase without a copy so the buffer's phases stay in step with its tiles
      mbar_expect_tx(&bars[s], 0u);
      return;
    }
    mbar_expect_tx(&bars[s], LY::TILE_BYTES);
    load_tile(buf0 + s * LY::TILE, &tmap, c0, 0, c2, 0, c4, &bars[s]);
  };
  if (tid == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    if ((int64_t)blockIdx.x < ntiles) issue(0, blockIdx.x);
    if ((int64_t)blockIdx.x + gridDim.x < ntiles) issue(1, blockIdx.x + gridDim.x);
  }
  __syncthreads();

  int kk = 0;
  for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x, ++kk) {
    const int s = kk & 1;
    const unsigned parity = (unsigned)((kk >> 1) & 1);
    float2* sm = buf0 + s * LY::TILE;
    int c0, c2, c4;
    coords(t, c0, c2, c4);
    // the wait acquires what thread 0 released when it armed the buffer: its s_active entry and the tile
    const bool staged = mbar_wait(&bars[s], parity);
    const bool active = s_active[s] != 0;
    // block-wide: every thread has read s_active[s] and seen the copy complete (thread 0 may re-arm after this)
    const bool ok = __syncthreads_and(staged ? 1 : 0) != 0;
    if (!ok) {
      if (tid == 0) {
        if (active) atomicOr(&const_cast<mmx_rhs_state*>(a.st + c4)->status, MMX_STATUS_TIMEOUT);
        mbar_wait(&bars[s], parity);  // drain the late copy before the buffer is re-armed
      }
    } else if (active) {
      using Plan = typename RegPlan<N>::type;
      if constexpr (OPS == OP_FWD) {
        RChain<-1, N, C, false, false, 1, Plan>::run(sm, smtw, nullptr, nullptr, 0, 0);
      } else if constexpr (OPS == OP_INV) {
        RChain<+1, N, C, false, false, 1, Plan>::run(sm, smtw, nullptr, nullptr, 0, 0);
      } else {
        const mmx_rhs_state* st = a.st + c4;
        const ChiCoef<float> cc = chi_coef<float>(st);
        const int64_t in0 = c0;
        if (tid < P) {
          const int64_t p = in0 + tid;
          float k1 = 0.f, k2 = 0.f;
          if (a.ndim == 3) {
            const int i1 = (int)(p / a.dims[2]);
            const int i2 = (int)(p - (int64_t)i1 * a.dims[2]);
            k1 = a.kv[1][i1];
            k2 = a.kv[2][i2];
          } else if (a.ndim == 2) {
            k1 = a.kv[1][p];
          }
          sk1[tid] = k1;
          sk2[tid] = k2;
        }
        // (the first stage's barriers publish the k tables before the Green stage reads them)
        const float ar = cc.alpha_re, ai = cc.alpha_im;
        if constexpr (C == 1) {
          using Init = typename PlanInit<Plan>::type;
          constexpr int RL = PlanLast<Plan>::value;
          RChain<-1, N, 1, false, false, 1, Init>::run(sm, smtw, nullptr, nullptr, 0, 0);
          green_fused_scalar<N, RL>(sm, smtw, sk0, sk1, sk2, ar, ai, ai * ai * a.inv_total, -ai * a.inv_total);
          RChain<+1, N, 1, false, false, RL, typename PlanReverse<Init>::type>::run(sm, smtw, nullptr, nullptr, 0, 0);
        } else {
          using GPlan = typename GreenPlan<N>::type;
          using Init = typename PlanInit<GPlan>::type;
          constexpr int RL = PlanLast<GPlan>::value;
          RChain<-1, N, 3, false, false, 1, Init>::run(sm, smtw, nullptr, nullptr, 0, 0);
          const float2 hs = divc(make_float2(0.f, ai), make_float2(ar, ai)) * a.inv_total;
          green_fused_vector<N, RL>(sm, smtw, sk0, sk1, sk2, in0 == 0 && c2 == 0, a.ndim, ar, ai,
                                    ai * ai * a.inv_total, -ai * a.inv_total, hs);
          RChain<+1, N, 3, false, false, RL, typename PlanReverse<Init>::type>::run(sm, smtw, nullptr, nullptr, 0, 0);
        }
      }
      // the stages end with a barrier; hand every thread's writes to the async proxy, then store the tile
      fence_async_smem();
      __syncthreads();
      if (tid == 0) store_tile(&tmap, c0, 0, c2, 0, c4, sm);
    }
    if (tid == 0) {
      const int64_t nxt = t + 2 * (int64_t)gridDim.x;
      if (nxt < ntiles) {
        stores_read_done();  // the store from this buffer has finished reading it
        issue(s, nxt);
      }
    }
  }
  if (tid == 0) stores_done();
}
