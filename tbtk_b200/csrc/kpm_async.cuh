// Recursion step for complex64 batches with per-thread asynchronous copies
// (cp.async, LDGSTS) into shared memory: one warp per row, the gathered rows
// of j_n and the row of j_{n-1} of the next S-1 rows in flight while the
// warp computes the current one.
//
// Why: in the register-staged kernel every gathered complex64 value in
// flight occupies a register, so at 128 registers a thread has two entries
// of one row in flight and a row costs several dependent round trips.  An
// asynchronous copy holds no register until it is read, so here the bytes
// in flight per SM are set by the shared-memory ring (S stages x (WMAX + 1)
// rows per warp), and the row's column indices and values are loaded one
// row further ahead again.  The per-element arithmetic and the entry order
// are those of kpm_step (Wide64: FP64 FMA on widened complex64 values), so
// vectors and directly gathered moments are bit-identical to it.
//
// Rows with more than WMAX entries take the rest from global memory;
// entries past the 32nd are loaded on demand.  No waits on other threads
// or flags: a warp only waits for its own copies (cp.async.wait_group).
#pragma once

#include "kpm_kernels.cuh"

namespace tbtkkpm {

__device__ __forceinline__ void cp_async_16(void *smem, const void *gmem) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(
                   (uint32_t)__cvta_generic_to_shared(smem)),
               "l"(gmem)
               : "memory");
}

__device__ __forceinline__ void cp_async_8(void *smem, const void *gmem) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(
                   (uint32_t)__cvta_generic_to_shared(smem)),
               "l"(gmem)
               : "memory");
}

__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}

template <int N> __device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Shared memory of one block: S stages x (WMAX gathered rows + the j_{n-1}
// row) x 32*VPT complex64 per warp.
template <int VPT, int S, int WMAX, int WPB> __host__ __device__ constexpr uint32_t async_smem_bytes() {
  return (uint32_t)(S * WPB * (WMAX + 1) * 32 * VPT * sizeof(float2));
}

// A row in the pipeline: its metadata (lane k holds entry k).
struct AsyncRow {
  uint32_t row, w;   // row index, slice width (entries incl. padding)
  uint32_t c;        // column of entry `lane` (kPad if none)
  double2 v;         // value of entry `lane`
  uint32_t valid;    // bit k: entry k < 32 is a real entry
  int diag;          // entry holding the row's own column, or -1
  bool ok, live;     // row inside the slices / inside the matrix
};

template <int VPT, bool FIRST, bool DOTS, int S, int WMAX, int WPB>
__global__ void __launch_bounds__(32 * WPB)
kpm_step_async(Sell A, uint32_t Bp, const float2 *__restrict__ x, float2 *__restrict__ y,
               Targets tg, uint32_t n_out, double2 *__restrict__ dots) {
  using V = float2;
  using AR = Wide64;
  using P = Pack<V, 32, VPT>;
  using L = typename P::L;
  using Acc = double2;
  constexpr int NL = P::NL;
  constexpr uint32_t kRow = 32 * VPT;  // complex64 per staged row
  constexpr unsigned full = 0xffffffffu;
  static_assert(WMAX <= 32, "staged entries come from one lane each");
  extern __shared__ __align__(16) unsigned char async_smem[];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  float2 *ring = reinterpret_cast<float2 *>(async_smem) + (size_t)wid * S * (WMAX + 1) * kRow;

  // rows of this warp: tile (blockIdx.x + i*gridDim.x), row wid of the tile
  const uint64_t ntiles = ((uint64_t)A.nslices * 32 + WPB - 1) / WPB;
  const uint32_t nrows =
      blockIdx.x < ntiles ? (uint32_t)((ntiles - 1 - blockIdx.x) / gridDim.x + 1) : 0u;

  auto load_meta = [&](uint32_t i) {
    AsyncRow m;
    const uint64_t r = ((uint64_t)blockIdx.x + (uint64_t)i * gridDim.x) * WPB + wid;
    m.row = (uint32_t)r;
    const uint32_t s = (uint32_t)(r >> 5), l = (uint32_t)(r & 31);
    m.ok = i < nrows && s < A.nslices;
    m.live = m.ok && r < A.N;
    m.w = 0;
    m.c = kPad;
    m.v = make_double2(0.0, 0.0);
    if (m.ok) {
      const uint32_t cb = __ldg(A.slice_ptr + s);
      m.w = __ldg(A.slice_ptr + s + 1) - cb;
      if ((uint32_t)lane < m.w) {
        const uint64_t slot = (uint64_t)(cb + lane) * 32 + l;
        m.c = __ldcs(A.col + slot);
        if (m.c != kPad) m.v = AR::value(A, slot);
      }
    }
    return m;
  };

  // Issues the copies of a row into its stage (every lane takes its chunks
  // of every gathered row) and closes the copy group.
  auto issue = [&](int stage, AsyncRow &m) {
    m.valid = __ballot_sync(full, m.c != kPad);
    const unsigned d = __ballot_sync(full, m.c == m.row && m.c != kPad);
    m.diag = d ? __ffs(d) - 1 : -1;
    if (m.ok) {
      float2 *st = ring + (size_t)stage * (WMAX + 1) * kRow;
      const uint32_t ns = min(m.w, (uint32_t)WMAX);
      for (uint32_t k = 0; k < ns; k++) {
        if (!((m.valid >> k) & 1u)) continue;
        const uint32_t ck = __shfl_sync(full, m.c, (int)k);
        const float2 *src = x + (uint64_t)ck * Bp;
        if constexpr (VPT == 1) {
          cp_async_8(st + k * kRow + lane, src + lane);
        } else {
#pragma unroll
          for (int q = 0; q < NL; q++)
            cp_async_16(reinterpret_cast<float4 *>(st + k * kRow) + q * 32 + lane,
                        reinterpret_cast<const float4 *>(src) + q * 32 + lane);
        }
      }
      if (!FIRST && m.live) {
        const float2 *src = y + (uint64_t)m.row * Bp;
        if constexpr (VPT == 1) {
          cp_async_8(st + WMAX * kRow + lane, src + lane);
        } else {
#pragma unroll
          for (int q = 0; q < NL; q++)
            cp_async_16(reinterpret_cast<float4 *>(st + WMAX * kRow) + q * 32 + lane,
                        reinterpret_cast<const float4 *>(src) + q * 32 + lane);
        }
      }
    }
    cp_async_commit();
  };

  double d_nn[DOTS ? VPT : 1], d_np[DOTS ? VPT : 1];
  if constexpr (DOTS) {
#pragma unroll
    for (int j = 0; j < VPT; j++) d_nn[j] = d_np[j] = 0.0;
  }

  auto compute = [&](int stage, const AsyncRow &m) {
    if (!m.ok) return;
    const float2 *st = ring + (size_t)stage * (WMAX + 1) * kRow;
    Acc acc[VPT];
    if constexpr (FIRST) {
#pragma unroll
      for (int j = 0; j < VPT; j++) acc[j] = Acc{0, 0};
    } else {
      L yr[NL];
      P::load_rw(st + WMAX * kRow, lane, yr);
#pragma unroll
      for (int j = 0; j < VPT; j++) {
        const Acc v = m.live ? P::get(yr, j) : Acc{0, 0};
        acc[j] = Acc{-v.x, -v.y};
      }
    }
    const uint32_t ns = min(m.w, (uint32_t)WMAX);
    for (uint32_t k = 0; k < ns; k++) {
      if (!((m.valid >> k) & 1u)) continue;
      double2 v;
      v.x = __shfl_sync(full, m.v.x, (int)k);
      v.y = __shfl_sync(full, m.v.y, (int)k);
      if constexpr (FIRST) v = AR::half(v);
      L raw[NL];
      P::load_rw(st + k * kRow, lane, raw);
#pragma unroll
      for (int j = 0; j < VPT; j++) acc[j] = AR::mac(acc[j], v, P::get(raw, j));
    }
    // entries past the staged ones, in order, from global memory
    for (uint32_t k = ns; k < m.w; k++) {
      uint32_t ck;
      double2 v;
      if (k < 32) {
        ck = __shfl_sync(full, m.c, (int)k);
        v.x = __shfl_sync(full, m.v.x, (int)k);
        v.y = __shfl_sync(full, m.v.y, (int)k);
      } else {
        const uint32_t s = m.row >> 5, l = m.row & 31;
        const uint64_t slot = (uint64_t)(__ldg(A.slice_ptr + s) + k) * 32 + l;
        ck = __ldcs(A.col + slot);
        v = ck != kPad ? AR::value(A, slot) : make_double2(0.0, 0.0);
      }
      if (ck == kPad) continue;
      if constexpr (FIRST) v = AR::half(v);
      L raw[NL];
      P::load(x + (uint64_t)ck * Bp, lane, raw);
#pragma unroll
      for (int j = 0; j < VPT; j++) acc[j] = AR::mac(acc[j], v, P::get(raw, j));
    }
    if (!m.live) return;
    const uint32_t row = m.row;
    if (target_hit(tg, row)) {
      for (uint32_t i = target_first(tg, row); i < tg.count && __ldg(tg.row + i) == row; i++) {
        const int jt = P::slot_of(lane, __ldg(tg.col + i));
        if (jt >= 0) {
#pragma unroll
          for (int j = 0; j < VPT; j++)
            if (j == jt) tg.mu[(uint64_t)__ldg(tg.out + i) * tg.ld + n_out] = acc[j];
        }
      }
    }
    float2 af[VPT];
#pragma unroll
    for (int j = 0; j < VPT; j++)
      af[j] = make_float2(__double2float_rn(acc[j].x), __double2float_rn(acc[j].y));
    P::storef(y + (uint64_t)row * Bp, lane, af);
    if constexpr (DOTS) {
      // j_n of this row: the staged diagonal entry, else a global load
      L self[NL];
      if (m.diag >= 0 && m.diag < WMAX) P::load_rw(st + m.diag * kRow, lane, self);
      else P::load(x + (uint64_t)row * Bp, lane, self);
#pragma unroll
      for (int j = 0; j < VPT; j++) {
        const float2 b = P::getf(self, j);
        d_nn[j] += (double)fmaf(af[j].x, af[j].x, af[j].y * af[j].y);
        d_np[j] += (double)fmaf(af[j].x, b.x, af[j].y * b.y);
      }
    }
  };

  AsyncRow ss[S];
  AsyncRow nm = load_meta(0);
#pragma unroll
  for (int u = 0; u < S - 1; u++) {
    ss[u] = nm;
    issue(u, ss[u]);
    nm = load_meta((uint32_t)u + 1);
  }
  for (uint32_t i0 = 0; i0 < nrows; i0 += S) {
#pragma unroll
    for (int u = 0; u < S; u++) {
      const int si = (u + S - 1) % S;
      ss[si] = nm;
      issue(si, ss[si]);
      nm = load_meta(i0 + (uint32_t)u + S);
      cp_async_wait<S - 1>();
      __syncwarp();
      compute(u, ss[u]);
      __syncwarp();
    }
  }
  cp_async_wait<0>();

  if constexpr (DOTS) {
    __shared__ double red[WPB][32][2];
#pragma unroll 1
    for (int j = 0; j < VPT; j++) {
      red[wid][lane][0] = d_nn[j];
      red[wid][lane][1] = d_np[j];
      __syncthreads();
      if (wid == 0) {
        double a = 0.0, b = 0.0;
        for (int q = 0; q < WPB; q++) {
          a += red[q][lane][0];
          b += red[q][lane][1];
        }
        double2 *o = dots + (uint64_t)blockIdx.x * 2 * Bp;
        const uint32_t c = P::col_of(lane, j);
        o[c] = make_double2(a, 0.0);
        o[Bp + c] = make_double2(b, 0.0);
      }
      __syncthreads();
    }
  }
}

}  // namespace tbtkkpm
