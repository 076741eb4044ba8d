// persist.cu - index files: the engine's bitmap slab, its level bounds and
// bin row counts, written and read in 64 MiB pieces through a pinned buffer.
// No counterpart in the reference, whose only on-disk state is the column
// files (ssb/cpuref.c:8-27).
#include <stdio.h>
#include <string.h>
#include <vector>
#include "engine.h"

namespace mb {
namespace {

constexpr uint32_t MBIX_VERSION = 1;
constexpr size_t CHUNK = 64ull << 20;

struct Fnv {  // FNV-1a, 64 bit
  uint64_t h = 0xcbf29ce484222325ull;
  void add(const void *p, size_t n) {
    const uint8_t *b = static_cast<const uint8_t *>(p);
    for (size_t i = 0; i < n; ++i) h = (h ^ b[i]) * 0x100000001b3ull;
  }
};

struct File {
  FILE *f = nullptr;
  Fnv fnv;
  ~File() {
    if (f) fclose(f);
  }
  bool put(const void *p, size_t n) {
    fnv.add(p, n);
    return fwrite(p, 1, n, f) == n;
  }
  bool get(void *p, size_t n) {
    if (fread(p, 1, n, f) != n) return false;
    fnv.add(p, n);
    return true;
  }
};

struct Pinned {
  void *p = nullptr;
  ~Pinned() {
    if (p) cudaFreeHost(p);
  }
};

}  // namespace
}  // namespace mb

using namespace mb;

extern "C" mb_status mb_engine_save_index(mb_engine *e, const char *path) {
  NvtxRange nvtx_("mb_engine_save_index");
  if (!e || !path) return fail(MB_ERR_INVALID, "mb_engine_save_index: NULL argument");
  Engine &E = e->E;
  if (!E.indexed) return fail(MB_ERR_INVALID, "mb_engine_save_index: no index built");
  MB_CUDA(cudaSetDevice(E.device));
  File F;
  F.f = fopen(path, "wb");
  if (!F.f) return fail(MB_ERR_IO, "mb_engine_save_index: cannot create %s", path);
  bool ok = F.put("MBIX", 4) && F.put(&MBIX_VERSION, 4) && F.put(&E.nrows, 8) && F.put(&E.stride, 8) &&
            F.put(&E.nbm, 4) && F.put(&E.level_mask, 4);
  for (auto &c : E.idx)
    for (auto &l : c.levels) {
      const uint32_t nb = l.nbins();
      ok = ok && F.put(&nb, 4) && F.put(l.bounds.data(), 8 * (nb + 1)) && F.put(l.pop.data(), 8 * nb);
    }
  Pinned buf;
  MB_CUDA(cudaMallocHost(&buf.p, CHUNK));
  const size_t total = (size_t)E.nbm * E.stride * 4;
  const uint8_t *src = reinterpret_cast<const uint8_t *>(E.islab);
  for (size_t off = 0; ok && off < total; off += CHUNK) {
    const size_t n = total - off < CHUNK ? total - off : CHUNK;
    MB_CUDA(cudaMemcpyAsync(buf.p, src + off, n, cudaMemcpyDeviceToHost, E.stream));
    MB_CUDA(cudaStreamSynchronize(E.stream));
    ok = F.put(buf.p, n);
  }
  const uint64_t h = F.fnv.h;
  ok = ok && fwrite(&h, 1, 8, F.f) == 8;
  if (!ok) return fail(MB_ERR_IO, "mb_engine_save_index: writing %s failed", path);
  return MB_OK;
}

extern "C" mb_status mb_engine_load_index(mb_engine *e, const char *path, uint32_t flags) {
  NvtxRange nvtx_("mb_engine_load_index");
  if (!e || !path) return fail(MB_ERR_INVALID, "mb_engine_load_index: NULL argument");
  if (flags & ~MB_INDEX_PROBE_DIMS) return fail(MB_ERR_INVALID, "mb_engine_load_index: flags 0x%x", flags);
  Engine &E = e->E;
  if (!E.custkey) return fail(MB_ERR_INVALID, "mb_engine_load_index: no table");
  MB_CUDA(cudaSetDevice(E.device));
  File F;
  F.f = fopen(path, "rb");
  if (!F.f) return fail(MB_ERR_IO, "mb_engine_load_index: cannot open %s", path);
  char magic[4];
  uint32_t ver = 0, nbm = 0, mask = 0;
  uint64_t nrows = 0, stride = 0;
  if (!F.get(magic, 4) || memcmp(magic, "MBIX", 4) != 0 || !F.get(&ver, 4) || ver != MBIX_VERSION)
    return fail(MB_ERR_IO, "mb_engine_load_index: %s is not an index file (version %u)", path, MBIX_VERSION);
  if (!F.get(&nrows, 8) || !F.get(&stride, 8) || !F.get(&nbm, 4) || !F.get(&mask, 4))
    return fail(MB_ERR_IO, "mb_engine_load_index: %s: short header", path);
  if (mask == 0 || (mask & ~MB_LEVELS_ALL))
    return fail(MB_ERR_INVALID, "mb_engine_load_index: %s: level mask 0x%x", path, mask);
  E.drop_index();
  MB_CUDA(cudaEventRecord(E.ev0, E.stream));
  if (flags & MB_INDEX_PROBE_DIMS) E.free_denorm();
  else MB_CHECK(E.build_denorm());
  E.level_mask = mask;
  MB_CHECK(E.setup_index_cols());  // the levels the file's index has
  uint32_t want = 0;
  for (auto &c : E.idx)
    for (auto &l : c.levels) want += l.nbins();
  if (nrows != E.nrows || stride != E.stride || nbm != want)
    return fail(MB_ERR_INVALID, "mb_engine_load_index: %s holds %llu rows x %u bitmaps, the table %llu x %u", path,
                (unsigned long long)nrows, nbm, (unsigned long long)E.nrows, want);
  for (auto &c : E.idx)
    for (auto &l : c.levels) {
      uint32_t nb = 0;
      std::vector<uint64_t> b, pop;
      bool ok = F.get(&nb, 4) && nb == l.nbins();
      if (ok) b.resize(nb + 1), pop.resize(nb);
      ok = ok && F.get(b.data(), 8 * (nb + 1)) && F.get(pop.data(), 8 * nb) && b == l.bounds;
      if (!ok) return fail(MB_ERR_INVALID, "mb_engine_load_index: %s: the levels of %s differ", path, c.name);
      l.pop = pop;
    }
  MB_CHECK(E.alloc((void **)&E.islab, (size_t)nbm * stride * 4));
  Pinned buf;
  MB_CUDA(cudaMallocHost(&buf.p, CHUNK));
  const size_t total = (size_t)nbm * stride * 4;
  uint8_t *dst = reinterpret_cast<uint8_t *>(E.islab);
  for (size_t off = 0; off < total; off += CHUNK) {
    const size_t n = total - off < CHUNK ? total - off : CHUNK;
    if (!F.get(buf.p, n)) {
      E.drop_index();
      return fail(MB_ERR_IO, "mb_engine_load_index: %s: short bitmap data", path);
    }
    MB_CUDA(cudaMemcpyAsync(dst + off, buf.p, n, cudaMemcpyHostToDevice, E.stream));
    MB_CUDA(cudaStreamSynchronize(E.stream));  // the pinned buffer is reused
  }
  const uint64_t h = F.fnv.h;
  uint64_t stored = 0;
  if (fread(&stored, 1, 8, F.f) != 8 || stored != h) {
    E.drop_index();
    return fail(MB_ERR_IO, "mb_engine_load_index: %s: hash mismatch", path);
  }
  uint64_t first = 0;
  for (auto &c : E.idx)
    for (auto &l : c.levels) {
      l.slab = E.islab + first * E.stride;
      first += l.nbins();
    }
  E.nbm = nbm;
  MB_CUDA(cudaEventRecord(E.ev1, E.stream));
  MB_CUDA(cudaStreamSynchronize(E.stream));
  cudaEventElapsedTime(&E.index_build_ms, E.ev0, E.ev1);
  E.indexed = true;
  return MB_OK;
}

// ------------------------------------------------------------ column files
extern "C" mb_status mb_write_column(const char *path, const void *host, uint64_t n, uint32_t width) {
  if (!path || (!host && n)) return fail(MB_ERR_INVALID, "mb_write_column: NULL argument");
  if (width != 1 && width != 2 && width != 4 && width != 8) return fail(MB_ERR_INVALID, "mb_write_column: width %u", width);
  FILE *f = fopen(path, "wb");
  if (!f) return fail(MB_ERR_IO, "mb_write_column: cannot create %s", path);
  bool ok = fwrite(&width, 4, 1, f) == 1 && (n == 0 || fwrite(host, width, n, f) == n);
  ok = (fclose(f) == 0) && ok;
  if (!ok) return fail(MB_ERR_IO, "mb_write_column: writing %s failed", path);
  return MB_OK;
}

namespace mb {
namespace {

// A device column of n elements of width `from` written as a column file of
// width `to` (values narrowed; the caller checked they fit), in pieces
// through a pinned buffer.
mb_status write_dev_column(Engine &E, const char *dir, const char *name, const void *dev, uint64_t n, uint32_t from,
                           uint32_t to) {
  char path[1024];
  snprintf(path, sizeof(path), "%s/%s", dir, name);
  FILE *f = fopen(path, "wb");
  if (!f) return fail(MB_ERR_IO, "mb_engine_save_ssb: cannot create %s", path);
  struct Closer {
    FILE *f;
    ~Closer() {
      if (f) fclose(f);
    }
  } closer{f};
  Pinned buf;
  MB_CUDA(cudaMallocHost(&buf.p, CHUNK));
  std::vector<uint8_t> out(CHUNK / from * to);
  bool ok = fwrite(&to, 4, 1, f) == 1;
  const uint64_t per = CHUNK / from;
  for (uint64_t i = 0; ok && i < n; i += per) {
    const uint64_t m = n - i < per ? n - i : per;
    MB_CUDA(cudaMemcpyAsync(buf.p, static_cast<const uint8_t *>(dev) + i * from, m * from, cudaMemcpyDeviceToHost,
                            E.stream));
    MB_CUDA(cudaStreamSynchronize(E.stream));
    const uint8_t *src = static_cast<const uint8_t *>(buf.p);
    if (from == to) {
      ok = fwrite(src, 1, m * to, f) == m * to;
      continue;
    }
    for (uint64_t j = 0; j < m; ++j) {
      uint64_t v = 0;
      memcpy(&v, src + j * from, from);
      memcpy(out.data() + j * to, &v, to);  // little-endian: the low bytes
    }
    ok = fwrite(out.data(), 1, m * to, f) == m * to;
  }
  closer.f = nullptr;
  ok = (fclose(f) == 0) && ok;
  if (!ok) return fail(MB_ERR_IO, "mb_engine_save_ssb: writing %s failed", path);
  return MB_OK;
}

}  // namespace
}  // namespace mb

extern "C" mb_status mb_engine_save_ssb(mb_engine *e, const char *dir) {
  if (!e || !dir) return fail(MB_ERR_INVALID, "mb_engine_save_ssb: NULL argument");
  Engine &E = e->E;
  if (!E.custkey) return fail(MB_ERR_INVALID, "mb_engine_save_ssb: no table");
  MB_CUDA(cudaSetDevice(E.device));
  // the reference's ssb_schema widths (ssb/ssbdemo.h:41-49)
  struct {
    const char *file, *col;
    const void *dev;
    uint32_t to;
  } fact[] = {{"loCustKey", "custkey", E.custkey, 4},         {"loPartKey", "partkey", E.partkey, 4},
              {"loOrderDate", "orderdate", E.orderdate, 2},   {"loExtendedPrice", "extendedprice", E.extendedprice, 4},
              {"loRevenue", "revenue", E.revenue, 4},         {"loSupplyCost", "supplycost", E.supplycost, 4},
              {"loSuppCity", "suppcity", E.suppcity, 1},      {"loQuantity", "quantity", E.quantity, 1},
              {"loDiscount", "discount", E.discount, 1}};
  for (auto &c : fact) MB_CHECK(write_dev_column(E, dir, c.file, c.dev, E.nrows, E.fact_width(c.col), c.to));
  const uint64_t nc = E.ncust + 1, np = E.npart + 1;
  MB_CHECK(write_dev_column(E, dir, "custCity", E.custcity, nc, 1, 1));
  MB_CHECK(write_dev_column(E, dir, "partMfgr", E.partmfgr, np, 2, 2));
  // the dimension attributes no query here reads: zeros of the same lengths
  std::vector<uint8_t> z(np * 2 > nc ? np * 2 : nc, 0);
  char path[1024];
  struct {
    const char *file;
    uint64_t n;
    uint32_t w;
  } zeros[] = {{"custMktSegment", nc, 1}, {"partName", np, 2},     {"partColor", np, 1},
               {"partType", np, 1},       {"partSize", np, 1},     {"partContainer", np, 1}};
  for (auto &c : zeros) {
    snprintf(path, sizeof(path), "%s/%s", dir, c.file);
    MB_CHECK(mb_write_column(path, z.data(), c.n, c.w));
  }
  return MB_OK;
}
