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
