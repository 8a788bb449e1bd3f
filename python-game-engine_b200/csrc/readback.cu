// Staging copy for host read-back of a field while the simulation keeps stepping.
//
// A game loop reads the density back every frame (common/simulation.py:322-324,
// get_density_field) while the next substep already rewrites it in place (the sources), so
// the field is first copied on the device into a staging buffer and the host copy runs from
// there on a copy stream. This copy runs between the substep kernels, whose multigrid solve
// keeps its working set in L2: here the loads and stores are cache-streaming (evict-first),
// so the staged field does not push that working set out of L2 before the next solve.
#include <algorithm>

#include "common.cuh"

namespace sg {

__global__ void k_stage_rows(int rows, int row_bytes, const unsigned char* __restrict__ src, int64_t lds,
                             unsigned char* __restrict__ dst, int64_t ldd) {
  // 16-byte units; the host has checked that pointers, strides and the row length allow them
  const int units = row_bytes >> 4;
  const int64_t n = (int64_t)rows * units;
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = q / units, u = q - r * units;
    const float4 v = __ldcs(reinterpret_cast<const float4*>(src + r * lds) + u);
    __stcs(reinterpret_cast<float4*>(dst + r * ldd) + u, v);
  }
}

}  // namespace sg

using namespace sg;

extern "C" {

int sg_stage_copy(int64_t rows, int64_t row_bytes, const void* src, int64_t ld_src_bytes, void* dst,
                  int64_t ld_dst_bytes, void* stream) {
  SG_REQUIRE(rows >= 0 && row_bytes >= 0 && rows < ((int64_t)1 << 31) && row_bytes < ((int64_t)1 << 31),
             "bad extent %lld x %lld bytes", (long long)rows, (long long)row_bytes);
  SG_REQUIRE(src && dst, "null pointer");
  SG_REQUIRE(ld_src_bytes >= row_bytes && ld_dst_bytes >= row_bytes, "row stride below row length");
  SG_REQUIRE(((uintptr_t)src | (uintptr_t)dst | (uint64_t)ld_src_bytes | (uint64_t)ld_dst_bytes |
              (uint64_t)row_bytes) % 16 == 0,
             "pointers, strides and row length must be multiples of 16 bytes");
  if (rows == 0 || row_bytes == 0) return SG_OK;
  const int64_t n = rows * (row_bytes / 16);
  const int blocks = (int)std::min<int64_t>((n + 255) / 256, 148 * 8);
  SG_LAUNCH(k_stage_rows<<<blocks, 256, 0, as_stream(stream)>>>((int)rows, (int)row_bytes,
                                                                 (const unsigned char*)src, ld_src_bytes,
                                                                 (unsigned char*)dst, ld_dst_bytes));
  return check_launch("sg_stage_copy");
}

}  // extern "C"

