// Builds the per-tile gather plans the tile-staged recursion steps read
// (kpm_tiled.cuh), on the device from the handle's scaled CSR.
#include "tbtkkpm.h"
#include "kpm_host.h"
#include "kpm_tiled.cuh"

#include <cub/cub.cuh>

#include <algorithm>

namespace tbtkkpm {

namespace {

template <int R>
int count_tiles(cudaStream_t st, const tbtkkpm_matrix *m, uint32_t ntiles, unsigned grid,
                DevBuf &tw, DevBuf &truns, DevBuf &tuniq, DevBuf &flags) {
  k_plan_count<R><<<grid, kPlanBlock, kPlanCap * 4, st>>>(
      m->N, ntiles, m->rowptr.as<uint32_t>(), m->col.as<uint32_t>(), tw.as<uint32_t>(),
      truns.as<uint32_t>(), tuniq.as<uint32_t>(), flags.as<unsigned>(), flags.as<unsigned>() + 2);
  return TBTKKPM_OK;
}

template <int R>
int pair_width(cudaStream_t st, const tbtkkpm_matrix *m, uint32_t ntiles, unsigned grid, DevBuf &tw,
               DevBuf &flags) {
  k_plan_pair_width<R><<<grid, kPlanBlock, 0, st>>>(m->N, ntiles, m->rowptr.as<uint32_t>(),
                                                     m->col.as<uint32_t>(), tw.as<uint32_t>(),
                                                     flags.as<unsigned>());
  return TBTKKPM_OK;
}

template <int R, bool CPLX, bool PAIRS = false>
int fill_tiles(cudaStream_t st, const tbtkkpm_matrix *m, uint32_t ntiles, unsigned grid,
               const DevBuf &ent, const DevBuf &run, const DevBuf &tw, const DevBuf &truns,
               const DevBuf &tuniq, TilePlanStore &p) {
  auto kern = k_plan_fill<R, CPLX, PAIRS>;
  constexpr int smem = 3 * kPlanCap * 4;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return cuda_fail(e, "tile plan: shared memory");
  kern<<<grid, kPlanBlock, smem, st>>>(
      m->N, ntiles, m->rowptr.as<uint32_t>(), m->col.as<uint32_t>(), m->val2.as<double2>(),
      ent.as<uint32_t>(), run.as<uint32_t>(), tw.as<uint32_t>(), truns.as<uint32_t>(),
      tuniq.as<uint32_t>(), p.hdr.as<uint4>(), p.runs.as<uint2>(), p.eslot.as<uint16_t>(),
      p.eval.ptr);
  return TBTKKPM_OK;
}

// pairs: the row-pair plan of complex values (R >= 16; k_plan_pair_width)
int build_plan(tbtkkpm_matrix *m, int R, bool cplx, bool pairs, TilePlanStore &p) {
  if (pairs && (!cplx || R < 16))
    return fail(TBTKKPM_ERR_UNSUPPORTED, "tile plan: row pairs need complex values and R >= 16");
  cudaStream_t st = m->stream;
  const uint32_t ntiles = (m->N + R - 1) / R;
  const unsigned grid = (unsigned)std::min<uint64_t>(ntiles, (uint64_t)sm_count(m->device) * 8);
  DevBuf tw, truns, tuniq, ent, run, flags, tmp;
  int rc;
  if ((rc = tw.reserve(4 * ((size_t)ntiles + 1))) || (rc = truns.reserve(4 * ((size_t)ntiles + 1))) ||
      (rc = tuniq.reserve(4 * ((size_t)ntiles + 1))) || (rc = ent.reserve(4 * ((size_t)ntiles + 1))) ||
      (rc = run.reserve(4 * ((size_t)ntiles + 1))) || (rc = flags.reserve(16)))
    return rc;
  cudaError_t e;
  if ((e = cudaMemsetAsync(flags.ptr, 0, 16, st)) ||
      (e = cudaMemsetAsync(tw.as<uint32_t>() + ntiles, 0, 4, st)) ||
      (e = cudaMemsetAsync(truns.as<uint32_t>() + ntiles, 0, 4, st)))
    return cuda_fail(e, "tile plan: staging");
  if (R == 8) rc = count_tiles<8>(st, m, ntiles, grid, tw, truns, tuniq, flags);
  else if (R == 16) rc = count_tiles<16>(st, m, ntiles, grid, tw, truns, tuniq, flags);
  else if (R == 32) rc = count_tiles<32>(st, m, ntiles, grid, tw, truns, tuniq, flags);
  else if (R == 64) rc = count_tiles<64>(st, m, ntiles, grid, tw, truns, tuniq, flags);
  else return fail(TBTKKPM_ERR_UNSUPPORTED, "tile plan: no builder for %d rows per tile", R);
  count_launches(1);
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "tile plan: count");
  if (pairs) {
    // entries per tile: the widest merge of a row pair instead of the widest row
    if ((e = cudaMemsetAsync(tw.ptr, 0, 4 * (size_t)ntiles, st))) return cuda_fail(e, "tile plan: pairs");
    if (R == 16) rc = pair_width<16>(st, m, ntiles, grid, tw, flags);
    else if (R == 32) rc = pair_width<32>(st, m, ntiles, grid, tw, flags);
    else rc = pair_width<64>(st, m, ntiles, grid, tw, flags);
    count_launches(1);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "tile plan: pairs");
  }
  // most distinct outside columns, widest row, a tile too large, widest pair merge
  unsigned hf[4] = {0, 0, 0, 0};
  if ((e = cudaMemcpyAsync(hf, flags.ptr, 16, cudaMemcpyDeviceToHost, st)) ||
      (e = cudaStreamSynchronize(st)))
    return cuda_fail(e, "tile plan: count");
  if (pairs) hf[1] = hf[3];
  p.ok = false;
  if (hf[2]) return TBTKKPM_OK;  // a tile past kPlanCap entries: no plan, other kernels run
  size_t tb = 0, tb2 = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, tb, tw.as<uint32_t>(), ent.as<uint32_t>(),
                                (int64_t)ntiles + 1, st);
  cub::DeviceScan::ExclusiveSum(nullptr, tb2, truns.as<uint32_t>(), run.as<uint32_t>(),
                                (int64_t)ntiles + 1, st);
  if ((rc = tmp.reserve(std::max<size_t>(std::max(tb, tb2), 16)))) return rc;
  cub::DeviceScan::ExclusiveSum(tmp.ptr, tb, tw.as<uint32_t>(), ent.as<uint32_t>(),
                                (int64_t)ntiles + 1, st);
  cub::DeviceScan::ExclusiveSum(tmp.ptr, tb2, truns.as<uint32_t>(), run.as<uint32_t>(),
                                (int64_t)ntiles + 1, st);
  uint32_t chunks = 0, nruns = 0;
  if ((e = cudaMemcpyAsync(&chunks, ent.as<uint32_t>() + ntiles, 4, cudaMemcpyDeviceToHost, st)) ||
      (e = cudaMemcpyAsync(&nruns, run.as<uint32_t>() + ntiles, 4, cudaMemcpyDeviceToHost, st)) ||
      (e = cudaStreamSynchronize(st)))
    return cuda_fail(e, "tile plan: scan");
  const size_t slots = std::max<size_t>((size_t)chunks * R, 8);
  const size_t vsz = cplx ? sizeof(double2) : sizeof(double);
  if ((rc = p.hdr.reserve(16 * (size_t)ntiles)) || (rc = p.runs.reserve(8 * std::max(nruns, 1u))) ||
      (rc = p.eslot.reserve(2 * slots)) || (rc = p.eval.reserve(vsz * slots)))
    return rc;
#define TBTKKPM_FILL(RR)                                                                      \
  (cplx ? fill_tiles<RR, true>(st, m, ntiles, grid, ent, run, tw, truns, tuniq, p)            \
        : fill_tiles<RR, false>(st, m, ntiles, grid, ent, run, tw, truns, tuniq, p))
  if (pairs) {
    if (R == 16) rc = fill_tiles<16, true, true>(st, m, ntiles, grid, ent, run, tw, truns, tuniq, p);
    else if (R == 32) rc = fill_tiles<32, true, true>(st, m, ntiles, grid, ent, run, tw, truns, tuniq, p);
    else rc = fill_tiles<64, true, true>(st, m, ntiles, grid, ent, run, tw, truns, tuniq, p);
  } else if (R == 8) rc = TBTKKPM_FILL(8);
  else if (R == 16) rc = TBTKKPM_FILL(16);
  else if (R == 32) rc = TBTKKPM_FILL(32);
  else rc = TBTKKPM_FILL(64);
#undef TBTKKPM_FILL
  if (rc) return rc;
  count_launches(1);
  if ((e = cudaGetLastError()) || (e = cudaStreamSynchronize(st)))
    return cuda_fail(e, "tile plan: fill");
  p.plan.hdr = p.hdr.as<uint4>();
  p.plan.runs = p.runs.as<uint2>();
  p.plan.eslot = p.eslot.as<uint16_t>();
  p.plan.eval = p.eval.ptr;
  p.plan.N = m->N;
  p.plan.ntiles = ntiles;
  p.plan.R = (uint32_t)R;
  p.plan.umax = hf[0];
  p.plan.wmax = hf[1];
  p.plan.nruns = nruns;
  p.plan.pairs = pairs ? 1u : 0u;
  p.ok = true;
  return TBTKKPM_OK;
}

}  // namespace

// The handle's plan for R-row tiles with real (cplx false) or complex
// values (pairs: the row-pair plan of complex values), built on first use;
// *out is null when the matrix has a tile the builder cannot take.
int tile_plan(tbtkkpm_matrix *m, int R, bool cplx, const TilePlan **out, bool pairs) {
  *out = nullptr;
  const int key = (pairs ? 1024 : 0) + 2 * R + (cplx ? 1 : 0);
  auto it = m->plans.find(key);
  if (it == m->plans.end()) {
    TilePlanStore &p = m->plans[key];
    int rc = build_plan(m, R, cplx, pairs, p);
    if (rc) {
      p.release();
      m->plans.erase(key);
      return rc;
    }
    it = m->plans.find(key);
  }
  if (it->second.ok) *out = &it->second.plan;
  return TBTKKPM_OK;
}

}  // namespace tbtkkpm
