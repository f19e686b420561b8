// Launcher of the fused-pair FP32 kernels (pairs.cuh).
#include <cuda_runtime.h>
#include <mutex>
#include "pairs.cuh"
#include "pairs.h"

namespace qcd {

namespace {

template <int MU, int BC, int KIND>
void* pair_fn() {
  return (void*)pair32<MU, BC, KIND>;
}

template <int MU, int BC>
void* pick_kind(int kind) {
  return kind == KIND_HB ? pair_fn<MU, BC, KIND_HB>() : kind == KIND_METRO ? pair_fn<MU, BC, KIND_METRO>()
                                                                        : pair_fn<MU, BC, KIND_OR>();
}
template <int MU>
void* pick_bc(int bc, int kind) {
  return bc == BC_PER ? pick_kind<MU, BC_PER>(kind) : bc == BC_PCC ? pick_kind<MU, BC_PCC>(kind)
                                                                   : pick_kind<MU, BC_PMC>(kind);
}
void* pick(int mu, int bc, int kind) {
  return mu == DIR_Y ? pick_bc<DIR_Y>(bc, kind) : mu == DIR_X ? pick_bc<DIR_X>(bc, kind) : pick_bc<DIR_T>(bc, kind);
}

// the shared-memory opt-in of each kernel, once per device
std::mutex g_attr_mu;
unsigned char g_attr_done[64][27];

cudaError_t opt_in(void* fn, int slot) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_attr_mu);
  if (g_attr_done[dev][slot]) return cudaSuccess;
  e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPairSmemBytes);
  if (e == cudaSuccess) g_attr_done[dev][slot] = 1;
  return e;
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
    cudaGetLastError();
  });
  return fn;
}

}  // namespace

cudaError_t pair_encode_maps(const float4* store, const Geo& g, PairMaps* out) {
  EncodeTiledFn enc = encode_fn();
  if (!enc) return cudaErrorNotSupported;
  // component (4 floats), y', x, t, class
  const cuuint64_t dims[5] = {4, (cuuint64_t)g.lyh, (cuuint64_t)g.lx, (cuuint64_t)g.lt, 6};
  const cuuint64_t strides[4] = {16, 16ull * g.lyh, 16ull * g.lyh * g.lx, 16ull * g.vh};
  const cuuint32_t elem[5] = {1, 1, 1, 1, 1};
  const cuuint32_t box_x[5] = {4, kPairW, kPairNR, 1, 1};
  const cuuint32_t box_t[5] = {4, kPairW, 1, kPairNR, 1};
  void* base = const_cast<float4*>(store);
  CUresult r = enc(&out->rows_x, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 5, base, dims, strides, box_x, elem,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r == CUDA_SUCCESS)
    r = enc(&out->rows_t, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 5, base, dims, strides, box_t, elem,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

int pair_segment(int ls, int tiles, int sms) {
  const int want = (8 * sms + tiles - 1) / tiles;  // segments for ~8 CTAs per SM
  int nseg = want < 1 ? 1 : want;
  const int most = ls / 16 < 1 ? 1 : ls / 16;
  if (nseg > most) nseg = most;
  return (ls + nseg - 1) / nseg;
}

cudaError_t pair_pass32(const float4* cur, float4* alt, const PairMaps& maps_cur, const PairMaps& maps_alt, const Geo& g,
                        int bc, int kind, const PhaseArgs& a, int seg, int sms, cudaStream_t stream) {
  PairPlanes P;
  for (int p = 0; p < 6; p++) P.src[p] = cur + (size_t)p * g.vh;
  P.alt_mask = 0;
  const int mus[3] = {DIR_Y, DIR_X, DIR_T};
  for (int m = 0; m < 3; m++) {
    const int mu = mus[m];
    P.dst_e = alt + (size_t)(mu * 2) * g.vh;
    P.dst_o = alt + (size_t)(mu * 2 + 1) * g.vh;
    int tr, ty, lrow, ls, nt;
    if (mu == DIR_Y) {
      tr = PairCfg<DIR_Y>::TR, ty = PairCfg<DIR_Y>::TY, lrow = g.lx, ls = g.lt, nt = PairCfg<DIR_Y>::NT;
    } else if (mu == DIR_X) {
      tr = PairCfg<DIR_X>::TR, ty = PairCfg<DIR_X>::TY, lrow = g.lx, ls = g.lt, nt = PairCfg<DIR_X>::NT;
    } else {
      tr = PairCfg<DIR_T>::TR, ty = PairCfg<DIR_T>::TY, lrow = g.lt, ls = g.lx, nt = PairCfg<DIR_T>::NT;
    }
    PairGrid pg;
    pg.n_row_tiles = (lrow + tr - 1) / tr;
    const int n_y_tiles = (g.lyh + ty - 1) / ty;
    const int tiles = pg.n_row_tiles * n_y_tiles;
    pg.seg = seg > 0 ? (seg < ls ? seg : ls) : pair_segment(ls, tiles, sms);
    const dim3 grid((unsigned int)tiles, (unsigned int)((ls + pg.seg - 1) / pg.seg));
    PhaseArgs am = a;
    am.phase_off = a.phase_off + (unsigned int)(2 * mu);
    void* fn = pick(mu, bc, kind);
    const int slot = mu * 9 + bc * 3 + (kind == KIND_HB ? 1 : kind == KIND_METRO ? 0 : 2);
    cudaError_t e = opt_in(fn, slot);
    if (e != cudaSuccess) return e;
    const CUtensorMap& tc = mu == DIR_T ? maps_cur.rows_t : maps_cur.rows_x;
    const CUtensorMap& ta = mu == DIR_T ? maps_alt.rows_t : maps_alt.rows_x;
    void* args[] = {(void*)&tc, (void*)&ta, (void*)&P, (void*)&g, (void*)&am, (void*)&pg};
    e = cudaLaunchKernel(fn, grid, dim3((unsigned int)nt), args, kPairSmemBytes, stream);
    if (e != cudaSuccess) return e;
    // the next pair reads this direction's new links from the other store
    P.src[mu * 2] = P.dst_e;
    P.src[mu * 2 + 1] = P.dst_o;
    P.alt_mask |= 3 << (mu * 2);
  }
  return cudaSuccess;
}

}  // namespace qcd
