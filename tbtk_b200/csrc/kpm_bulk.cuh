// Recursion step for wide batches with bulk asynchronous copies (sm_90+,
// used on sm_100a): one warp per row, the gathered rows of j_n and the row of
// j_{n-1} staged in shared memory by cp.async.bulk with mbarrier completion.
//
// Why: for a batch of B complex64 vectors every matrix entry of a row needs
// a B*8-byte row of j_n.  Loading those into registers caps how many rows a
// thread can have in flight (the register file holds them), and each row
// then costs several dependent round trips.  Here one lane issues one bulk
// copy per gathered row into a per-warp ring of S stages; the warp computes
// row i from shared memory while rows i+1 .. i+S-1 are in flight, so the
// bytes in flight per SM are set by the ring size, not by registers.
// Only non-multicast bulk loads are issued.
//
// Every wait on an mbarrier is bounded; a wait that runs out sets *err to
// kErrTimeout, drains the copies the warp has in flight (bounded again) and
// leaves the loop, so a kernel never spins forever.
#pragma once

#include "kpm_kernels.cuh"

namespace tbtkkpm {

constexpr int kBulkWMax = 12;            // entries per row staged in the ring
constexpr uint32_t kWaitLimit = 1u << 22; // try_wait polls before giving up
constexpr int kErrTimeout = 1;

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bulk copy global -> this CTA's shared memory, completing on `bar`.
// dst and src 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes,
                                          uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// Bounded wait of the whole warp for phase `parity` of `bar`.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity) {
  for (uint32_t it = 0; it < kWaitLimit; it++)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// One ring stage: barrier, the row's entries, then (kBulkWMax + 1) rows of
// Bp values (entries 0..kBulkWMax-1 gathered from j_n, slot kBulkWMax holds
// j_{n-1} of the row).
struct StageMeta {
  uint64_t bar;
  uint32_t row, w, nvalid, hit;
  uint32_t col[kBulkWMax];
  double2 val[kBulkWMax];
};
constexpr uint32_t kStageMetaBytes = (sizeof(StageMeta) + 127) / 128 * 128;
static_assert(kStageMetaBytes == 384, "gen_steps.py assumes 384-byte stage headers");

template <typename V, int VPT>
__host__ __device__ constexpr uint32_t bulk_stage_bytes() {
  return kStageMetaBytes + (kBulkWMax + 1) * 32u * VPT * (uint32_t)sizeof(V);
}

template <typename V, int VPT, int S, int WPB>
__host__ __device__ constexpr uint32_t bulk_smem_bytes() {
  return S * WPB * bulk_stage_bytes<V, VPT>();
}

// Step kernel (same recursion and outputs as kpm_step, TPR = 32): warp w
// of the grid owns rows w, w + W, w + 2W, ... (W = warps in the grid).
template <typename V, typename AR, int VPT, bool FIRST, bool DOTS, int S, int WPB>
__global__ void __launch_bounds__(32 * WPB)
kpm_step_bulk(Sell A, uint32_t Bp, const V *__restrict__ x, V *__restrict__ y, Targets tg,
              uint32_t n_out, double2 *__restrict__ dots, int *err) {
  using Acc = typename AR::Acc;
  using P = Pack<V, 32, VPT>;
  using L = typename P::L;
  constexpr int NL = P::NL;
  extern __shared__ __align__(128) unsigned char smem[];
  constexpr uint32_t SB = bulk_stage_bytes<V, VPT>();
  constexpr uint32_t ROWB = 32u * VPT * sizeof(V);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  unsigned char *ring = smem + (size_t)wid * S * SB;
  auto meta = [&](int s) { return reinterpret_cast<StageMeta *>(ring + (size_t)s * SB); };
  auto data = [&](int s, int k) {
    return reinterpret_cast<V *>(ring + (size_t)s * SB + kStageMetaBytes + (size_t)k * ROWB);
  };
  const uint32_t nrows = A.nslices * 32;
  const uint32_t W = gridDim.x * WPB;
  const uint32_t gw = blockIdx.x * WPB + wid;
  double2 d_nn[DOTS ? VPT : 1], d_np[DOTS ? VPT : 1];
  if constexpr (DOTS) {
#pragma unroll
    for (int j = 0; j < VPT; j++) d_nn[j] = d_np[j] = make_double2(0.0, 0.0);
  }
  if (lane == 0)
    for (int s = 0; s < S; s++) mbar_init(&meta(s)->bar, 1);
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  __syncwarp();
  uint32_t phase = 0;  // bit s: parity to wait for on stage s

  // A row's entries, loaded one iteration before its copies are issued
  // (lane k holds entry k), so the slice-pointer -> column-index chain is
  // off the critical path.
  struct RowMeta {
    uint32_t r, w, c, hit;
    double2 v;
  };
  auto load_meta = [&](uint32_t i) {
    RowMeta m;
    m.r = gw + i * W;
    const uint32_t sl = m.r >> 5, l = m.r & 31;
    const uint32_t cb = __ldg(A.slice_ptr + sl);
    m.w = __ldg(A.slice_ptr + sl + 1) - cb;
    m.c = kPad;
    m.v = make_double2(0.0, 0.0);
    if ((uint32_t)lane < m.w && lane < kBulkWMax) {
      m.c = __ldcs(A.col + (uint64_t)(cb + lane) * 32 + l);
      if (m.c != kPad) m.v = __ldcs(A.val + (uint64_t)(cb + lane) * 32 + l);
    }
    m.hit = (lane == 0 && m.r < A.N) ? (uint32_t)target_hit(tg, m.r) : 0u;
    return m;
  };
  // Issues the copies of the i-th row of this warp into stage i % S.
  auto issue = [&](const RowMeta &m, uint32_t i) {
    const int s = (int)(i % S);
    StageMeta *mt = meta(s);
    const bool live = m.r < A.N;
    const unsigned valid = __ballot_sync(0xffffffffu, m.c != kPad);
    const uint32_t nvalid = __popc(valid);
    const uint32_t bytes = (nvalid + ((!FIRST && live) ? 1u : 0u)) * ROWB;
    if (lane < kBulkWMax) {
      mt->col[lane] = m.c;
      mt->val[lane] = m.v;
    }
    if (lane == 0) {
      mt->row = m.r;
      mt->w = m.w;
      mt->nvalid = nvalid;
      mt->hit = m.hit;
      mbar_expect_tx(&mt->bar, bytes);
    }
    __syncwarp();
    if (m.c != kPad) bulk_load(data(s, lane), x + (uint64_t)m.c * Bp, ROWB, &mt->bar);
    if (!FIRST && live && lane == 31)
      bulk_load(data(s, kBulkWMax), y + (uint64_t)m.r * Bp, ROWB, &mt->bar);
  };

  const uint32_t mine = gw < nrows ? (nrows - gw + W - 1) / W : 0;
  for (uint32_t i = 0; i + 1 < (uint32_t)S && i < mine; i++) issue(load_meta(i), i);
  RowMeta pending;
  if ((uint32_t)S - 1 < mine) pending = load_meta(S - 1);
  bool failed = false;
  uint32_t i = 0;
  for (; i < mine; i++) {
    if (i + S - 1 < mine) {
      const RowMeta m = pending;
      if (i + S < mine) pending = load_meta(i + S);
      issue(m, i + S - 1);
    }
    const int s = (int)(i % S);
    StageMeta *mt = meta(s);
    if (!mbar_wait_bounded(&mt->bar, (phase >> s) & 1u)) {
      failed = true;
      break;
    }
    phase ^= 1u << s;
    const uint32_t r = mt->row, w = mt->w;
    if (r < A.N) {
      Acc acc[VPT];
      if constexpr (FIRST) {
#pragma unroll
        for (int j = 0; j < VPT; j++) acc[j] = Acc{0, 0};
      } else {
        L yr[NL];
        P::load_rw(data(s, kBulkWMax), lane, yr);
#pragma unroll
        for (int j = 0; j < VPT; j++) {
          const double2 v = P::get(yr, j);
          acc[j] = Acc{-v.x, -v.y};
        }
      }
      int self = -1;
      const uint32_t ws = min(w, (uint32_t)kBulkWMax);
      for (uint32_t k = 0; k < ws; k++) {
        const uint32_t c = mt->col[k];
        if (c == kPad) continue;
        double2 v = mt->val[k];
        if constexpr (FIRST) v = AR::half(v);
        L xr[NL];
        P::load_rw(data(s, (int)k), lane, xr);
#pragma unroll
        for (int j = 0; j < VPT; j++) acc[j] = AR::mac(acc[j], v, P::get(xr, j));
        if (c == r) self = (int)k;
      }
      // entries past the staged ones (rows wider than kBulkWMax)
      if (w > (uint32_t)kBulkWMax) {
        const uint32_t sl = r >> 5, l = r & 31, cb = __ldg(A.slice_ptr + sl);
        for (uint32_t k = kBulkWMax; k < w; k++) {
          const uint32_t c = __ldcs(A.col + (uint64_t)(cb + k) * 32 + l);
          if (c == kPad) continue;
          double2 v = AR::value(A, (uint64_t)(cb + k) * 32 + l);
          if constexpr (FIRST) v = AR::half(v);
          L xr[NL];
          P::load(x + (uint64_t)c * Bp, lane, xr);
#pragma unroll
          for (int j = 0; j < VPT; j++) acc[j] = AR::mac(acc[j], v, P::get(xr, j));
        }
      }
      if (mt->hit) {
        for (uint32_t t = target_first(tg, r); t < tg.count && __ldg(tg.row + t) == r; t++) {
          const int jt = P::slot_of(lane, __ldg(tg.col + t));
          if (jt >= 0) {
#pragma unroll
            for (int j = 0; j < VPT; j++)
              if (j == jt) tg.mu[(uint64_t)__ldg(tg.out + t) * tg.ld + n_out] = AR::wide(acc[j]);
          }
        }
      }
      P::store(y + (uint64_t)r * Bp, lane, acc);  // acc now holds the values as stored
      if constexpr (DOTS) {
        L sr[NL];
        if (self >= 0) P::load_rw(data(s, self), lane, sr);
        else P::load(x + (uint64_t)r * Bp, lane, sr);
#pragma unroll
        for (int j = 0; j < VPT; j++) {
          const double2 a = AR::wide(acc[j]);
          const double2 b = P::get(sr, j);
          d_nn[j].x = fma(a.x, a.x, fma(a.y, a.y, d_nn[j].x));
          d_np[j].x = fma(a.x, b.x, fma(a.y, b.y, d_np[j].x));
          d_np[j].y = fma(a.x, b.y, fma(-a.y, b.x, d_np[j].y));
        }
      }
    }
    __syncwarp();  // the stage is read; it may be refilled
  }
  if (failed) {
    if (lane == 0) atomicExch(err, kErrTimeout);
    // drain the copies still in flight into this warp's ring, the stage that
    // ran out included
    for (uint32_t j = i; j < mine && j < i + (uint32_t)S; j++) {
      const int s = (int)(j % S);
      mbar_wait_bounded(&meta(s)->bar, (phase >> s) & 1u);
    }
  }
  if constexpr (DOTS) {
    // per-warp partials, then a fixed-order sum over the block's warps
    __shared__ double2 red[WPB][32][2];
#pragma unroll 1
    for (int j = 0; j < VPT; j++) {
      red[wid][lane][0] = d_nn[j];
      red[wid][lane][1] = d_np[j];
      __syncthreads();
      if (wid == 0) {
        double2 a = make_double2(0.0, 0.0), b = make_double2(0.0, 0.0);
        for (int q = 0; q < WPB; q++) {
          a.x += red[q][lane][0].x;
          b.x += red[q][lane][1].x;
          b.y += red[q][lane][1].y;
        }
        double2 *o = dots + (uint64_t)blockIdx.x * 2 * Bp;
        const uint32_t c = P::col_of(lane, j);
        o[c] = a;
        o[Bp + c] = b;
      }
      __syncthreads();
    }
  }
}

}  // namespace tbtkkpm
