// gen.cu - seeded, counter-based synthetic data generation on the device.
//
// Every value is a pure function of (seed, column, row) (merle_b200_gen.h), so
// tables of any size are generated in place in HBM with one grid-stride pass
// per table and no host transfer.  The CPU oracle calls the same inline
// functions and sees identical values.
#include "common.cuh"
#include "merle_b200_gen.h"

namespace mb {

__global__ void gen_flat_kernel(uint64_t seed, uint64_t row0, uint64_t n, int32_t *a,
                                int32_t *b, int32_t *c, int32_t *d, int32_t *e) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t r = row0 + i;
    if (a) a[i] = mbg_flat_a(seed, r);
    if (b) b[i] = mbg_flat_b(seed, r);
    if (c) c[i] = mbg_flat_c(seed, r);
    if (d) d[i] = mbg_flat_d(seed, r);
    if (e) e[i] = mbg_flat_e(seed, r);
  }
}

__device__ __forceinline__ void put(void *p, uint64_t i, uint32_t v, uint32_t w) {
  if (!p) return;
  if (w == 1) reinterpret_cast<uint8_t *>(p)[i] = (uint8_t)v;
  else if (w == 2) reinterpret_cast<uint16_t *>(p)[i] = (uint16_t)v;
  else reinterpret_cast<uint32_t *>(p)[i] = v;
}

__global__ void gen_star_kernel(uint64_t seed, uint32_t k, uint64_t row0, uint64_t n,
                                int width4, mb_star_cols o) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    mbg_lorow r = mbg_star_row(seed, k, row0 + i);
    put(o.custkey, i, r.custkey, 4);
    put(o.partkey, i, r.partkey, 4);
    put(o.suppkey, i, r.suppkey, 4);
    put(o.orderdate, i, r.orderdate, width4 ? 4 : 2);
    put(o.quantity, i, r.quantity, width4 ? 4 : 1);
    put(o.discount, i, r.discount, width4 ? 4 : 1);
    put(o.extendedprice, i, r.extendedprice, 4);
    put(o.revenue, i, r.revenue, 4);
    put(o.supplycost, i, r.supplycost, 4);
    put(o.suppcity, i, r.suppcity, width4 ? 4 : 1);
  }
}

__global__ void gen_dims_kernel(uint64_t seed, uint64_t nc, uint64_t ns, uint64_t np,
                                uint8_t *cc, uint8_t *sc, uint16_t *pm) {
  uint64_t total = (nc + 1) + (ns + 1) + (np + 1);
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total;
       i += (uint64_t)gridDim.x * blockDim.x) {
    if (i <= nc) {
      if (cc) cc[i] = (uint8_t)mbg_cust_city(seed, i);
    } else if (i <= nc + 1 + ns) {
      uint64_t key = i - (nc + 1);
      if (sc) sc[key] = (uint8_t)mbg_supp_city(seed, key);
    } else {
      uint64_t key = i - (nc + 1) - (ns + 1);
      if (pm) pm[key] = (uint16_t)mbg_part_mfgr(seed, key);
    }
  }
}

static unsigned gen_grid(uint64_t n) {
  uint64_t g = ceil_div(n, 256);
  uint64_t cap = (uint64_t)dev_info().sms * 16;
  return (unsigned)(g < cap ? (g ? g : 1) : cap);
}

}  // namespace mb

using namespace mb;

extern "C" mb_status mb_gen_flat(uint64_t seed, uint64_t row0, uint64_t n, int32_t *a,
                                 int32_t *b, int32_t *c, int32_t *d, int32_t *e,
                                 void *stream) {
  if (n == 0) return MB_OK;
  gen_flat_kernel<<<gen_grid(n), 256, 0, as_stream(stream)>>>(seed, row0, n, a, b, c, d, e);
  MB_LAUNCH_CHECK("gen_flat_kernel");
  return MB_OK;
}

extern "C" mb_status mb_gen_star(uint64_t seed, uint32_t k, uint64_t row0, uint64_t n,
                                 int width4, const mb_star_cols *out, void *stream) {
  if (!out || k == 0) return fail(MB_ERR_INVALID, "mb_gen_star: out is NULL or k == 0");
  if (n == 0) return MB_OK;
  gen_star_kernel<<<gen_grid(n), 256, 0, as_stream(stream)>>>(seed, k, row0, n, width4, *out);
  MB_LAUNCH_CHECK("gen_star_kernel");
  return MB_OK;
}

extern "C" mb_status mb_gen_star_dims(uint64_t seed, uint32_t k, uint8_t *custcity,
                                      uint8_t *suppcity, uint16_t *partmfgr, void *stream) {
  if (k == 0) return fail(MB_ERR_INVALID, "mb_gen_star_dims: k == 0");
  uint64_t nc = mbg_star_ncust(k), ns = mbg_star_nsupp(k), np = mbg_star_npart(k);
  gen_dims_kernel<<<gen_grid(nc + ns + np + 3), 256, 0, as_stream(stream)>>>(
      seed, nc, ns, np, custcity, suppcity, partmfgr);
  MB_LAUNCH_CHECK("gen_dims_kernel");
  return MB_OK;
}
