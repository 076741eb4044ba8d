// legacy.cu - the reference's own C entry points (ssb_*, synth_*,
// window_zipf) over this library's kernels, so a driver written against
// ssb/ssbdemo.h and synth/synthdemo.h links against libmerleb200.so as is.
//
// Each entry point does what its reference counterpart does (cited per
// function) with the mb_* kernels: one-pass bin creation, the fused program +
// join-probe + group-by kernel, the materialised three-stage plan, the
// no-index join.  Results are the reference's uint32 values (the int64 sums
// truncated).  Errors print one line to stderr and return 0 / NULL / false
// instead of exiting.
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <vector>
#include "engine.h"
#include "merle_b200_legacy.h"

// Bin boundaries of the fixed SSB index (ssb/bmpidx-create.cu:8-30): callers
// read these tables, so they keep the reference's values.
const uint64_t dateSpBin[8] = {SSBDATE_920101, SSBDATE_930101, SSBDATE_940101, SSBDATE_950101,
                               SSBDATE_960101, SSBDATE_970101, SSBDATE_980101, SSBDATE_990101};
const uint64_t dateDeBin[5] = {SSBDATE_940101, SSBDATE_940201, SSBDATE_940301, SSBDATE_971201, SSBDATE_980101};
const uint64_t discntSpBin[5] = {0, 2, 5, 8, 11};
const uint64_t discntDeBin[12] = {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11};
const uint64_t qtySpBin[6] = {1, 11, 21, 31, 41, 51};
const uint64_t qtyDeBin[11] = {1, 6, 11, 16, 21, 26, 31, 36, 41, 46, 51};
const uint64_t mfgrSpBin[6] = {0, 200, 400, 600, 800, 1000};
const uint64_t mfgrDeBin[6] = {40, 80, 120, 160, 240, 280};
const uint64_t sCitySpBin[6] = {0, 50, 100, 150, 200, 250};
const uint64_t sCityDeBin[4] = {50, 60, 190, 200};

namespace mb {
namespace {

// ------------------------------------------------------------ files
// One column file: a 4-byte element-width header, then the raw array
// (ssb/cpuref.c:8-27).  bytes == 0: the array is the rest of the file.
bool read_col(const char *dir, const char *name, size_t bytes, void **out, size_t *got) {
  *out = nullptr;
  char path[1024];
  snprintf(path, sizeof(path), "%s/%s", dir, name);
  FILE *f = fopen(path, "rb");
  if (!f) {
    fprintf(stderr, "merle_b200: cannot open %s\n", path);
    return false;
  }
  bool ok = fseek(f, 0, SEEK_END) == 0;
  const long len = ok ? ftell(f) : -1;
  ok = ok && len >= 4;
  if (ok && bytes == 0) bytes = (size_t)len - 4;
  ok = ok && (size_t)len - 4 >= bytes && fseek(f, 4, SEEK_SET) == 0;
  void *p = ok ? malloc(bytes ? bytes : 1) : nullptr;
  ok = ok && p && fread(p, 1, bytes, f) == bytes;
  fclose(f);
  if (!ok) {
    free(p);
    fprintf(stderr, "merle_b200: cannot read %zu bytes of %s\n", bytes, path);
    return false;
  }
  *out = p;
  if (got) *got = bytes;
  return true;
}

void *to_dev(const void *h, size_t bytes) {
  void *d = nullptr;
  if (cudaMalloc(&d, bytes ? bytes : 1) != cudaSuccess) return nullptr;
  if (bytes && cudaMemcpy(d, h, bytes, cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaFree(d);
    return nullptr;
  }
  return d;
}

__global__ void trunc32_kernel(const int64_t *in, uint32_t *out, uint32_t n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    out[i] = (uint32_t)(uint64_t)in[i];
}

void trunc32(const int64_t *in, uint32_t *out, uint32_t n) {
  if (n) trunc32_kernel<<<(n + 255) / 256, 256>>>(in, out, n);
}

mb_src src_of(const void *col, uint32_t w, const uint32_t *fk = nullptr, uint64_t dimsz = 0) {
  mb_src s;
  memset(&s, 0, sizeof(s));
  s.col = col, s.fk = fk, s.dimsz = dimsz, s.width = w;
  return s;
}

// Device buffers freed at scope exit.
struct DevBufs {
  std::vector<void *> p;
  void *get(size_t bytes) {
    void *d = nullptr;
    if (cudaMalloc(&d, bytes ? bytes : 1) != cudaSuccess) return nullptr;
    p.push_back(d);
    return d;
  }
  ~DevBufs() {
    cudaDeviceSynchronize();
    for (void *d : p) cudaFree(d);
  }
};

struct Timer {
  cudaEvent_t a = nullptr, b = nullptr;
  Timer() {
    cudaEventCreate(&a);
    cudaEventCreate(&b);
  }
  ~Timer() {
    cudaEventDestroy(a);
    cudaEventDestroy(b);
  }
  void start() { cudaEventRecord(a); }
  float stop() {
    float ms = 0;
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    cudaEventElapsedTime(&ms, a, b);
    return ms;
  }
};

// ------------------------------------------------------------ SSB queries
// The 13 parameterisations of ssb_cpujoin / ssb_bmp_fixed
// (ssb/cpuref.c:248-298, ssb/fixedlayout.cu:145-186), in result order.  Q1.1
// takes quantity [1, 25) as the index paths do (ssb/fixedlayout.cu:150; the
// host path's [0, 25) selects the same rows: quantities start at 1).
struct SsbQ {
  const char *name;
  mb_query q;
};
const SsbQ SSB13[13] = {
    {"SSB11", {1, {SSBDATE_930101, SSBDATE_940101, 1, 4, 1, 25}}},
    {"SSB12", {1, {SSBDATE_940101, SSBDATE_940201, 4, 7, 26, 36}}},
    {"SSB13", {1, {SSBDATE_940204, SSBDATE_940211, 5, 8, 26, 36}}},
    {"SSB21", {2, {40, 80, 150, 200}}},
    {"SSB22", {2, {260, 268, 200, 250}}},
    {"SSB23", {2, {260, 261, 50, 100}}},
    {"SSB31", {3, {200, 250, 200, 250, SSBDATE_920101, SSBDATE_980101}}},
    {"SSB32", {3, {190, 200, 190, 200, SSBDATE_920101, SSBDATE_980101}}},
    {"SSB33", {3, {51, 55, 51, 55, SSBDATE_920101, SSBDATE_980101}}},
    {"SSB34", {3, {51, 55, 51, 55, SSBDATE_971201, SSBDATE_980101}}},
    {"SSB41", {4, {150, 200, 150, 200, 0, 400, SSBDATE_920101, SSBDATE_990101}}},
    {"SSB42", {4, {150, 200, 150, 200, 0, 400, SSBDATE_970101, SSBDATE_990101}}},
    {"SSB43", {4, {150, 200, 190, 200, 120, 160, SSBDATE_970101, SSBDATE_990101}}},
};

uint32_t ssb_offset(int i) {
  uint32_t o = 0;
  for (int j = 0; j < i; ++j) o += query_ngroups(SSB13[j].q);
  return o;
}

// The ops over a device ssb_schema (the reference's dimension probes carry no
// bound check: dimsz 0).
SsbSrc ssb_srcs(const ssb_schema *d) {
  SsbSrc S;
  S.date = src_of(d->loOrderDate, 2);
  S.disc = src_of(d->loDiscount, 1);
  S.qty = src_of(d->loQuantity, 1);
  S.eprice = src_of(d->loExtendedPrice, 4);
  S.rev = src_of(d->loRevenue, 4);
  S.scost = src_of(d->loSupplyCost, 4);
  S.scity = src_of(d->loSuppCity, 1);
  S.ccity = src_of(d->custCity, 1, d->loCustKey);
  S.mfgr = src_of(d->partMfgr, 2, d->loPartKey);
  return S;
}

// A program over the fixed index in one of the reference's three layouts
// (0 sparse, 1 medium, 2 dense: which columns take the fine bins,
// ssb/fixedlayout.cu:37-143).
struct FixedPrg {
  mb_vprg p;
  const uint32_t *mid[MB_MAXCOLS][MB_MAXBINS];
};

#define NB(a) (uint32_t)(sizeof(a) / sizeof((a)[0]))
bool cover(const ssb_bmp *b, char col, bool dense, uint64_t lo, uint64_t hi, mb_col *out, const uint32_t **mid) {
  const uint32_t *const *sp, *const *de;
  const uint64_t *spb, *deb;
  uint32_t ns, nd;
  switch (col) {
  case 'd': sp = b->dateSparse, ns = NB(b->dateSparse), spb = dateSpBin, de = b->dateDense, nd = NB(b->dateDense), deb = dateDeBin; break;
  case 'i': sp = b->discntSparse, ns = NB(b->discntSparse), spb = discntSpBin, de = b->discntDense, nd = NB(b->discntDense), deb = discntDeBin; break;
  case 'q': sp = b->qtySparse, ns = NB(b->qtySparse), spb = qtySpBin, de = b->qtyDense, nd = NB(b->qtyDense), deb = qtyDeBin; break;
  case 'm': sp = b->mfgrSparse, ns = NB(b->mfgrSparse), spb = mfgrSpBin, de = b->mfgrDense, nd = NB(b->mfgrDense), deb = mfgrDeBin; break;
  case 's': sp = b->sCitySparse, ns = NB(b->sCitySparse), spb = sCitySpBin, de = b->sCityDense, nd = NB(b->sCityDense), deb = sCityDeBin; break;
  default: sp = b->cCitySparse, ns = NB(b->cCitySparse), spb = sCitySpBin, de = b->cCityDense, nd = NB(b->cCityDense), deb = sCityDeBin; break;
  }
  const mb_status st = dense ? mb_col_from_bin2(ns, sp, spb, nd, de, deb, lo, hi, out, mid)
                             : mb_col_from_bin(ns, sp, spb, lo, hi, out, mid);
  return st == MB_OK;
}

bool fixed_prg(const ssb_bmp *b, const mb_query &q, uint64_t n, int layout, FixedPrg &F) {
  memset(&F, 0, sizeof(F));
  mb_vprg &p = F.p;
  p.factsz = n;
  const uint32_t *a = q.p;
  auto ins = [&](int i, uint32_t op, uint32_t d, uint32_t s1, uint32_t s2) {
    p.instrs[i].opcode = op, p.instrs[i].dstreg = d, p.instrs[i].src1 = s1, p.instrs[i].src2 = s2;
  };
  bool ok = true;
  if (q.tmpl == 1) {
    p.ncols = 3;
    ok = cover(b, 'd', layout >= 2, a[0], a[1], &p.cols[0], F.mid[0]) &&
         cover(b, 'i', layout >= 1, a[2], a[3], &p.cols[1], F.mid[1]) &&
         cover(b, 'q', layout >= 1, a[4], a[5], &p.cols[2], F.mid[2]);
    ins(0, MB_ORM, 0, 0, 0), ins(1, MB_ANDM, 0, 1, 0), ins(2, MB_ANDM, 0, 2, 0);
  } else if (q.tmpl == 2) {
    p.ncols = 2;
    ok = cover(b, 'm', layout >= 1, a[0], a[1], &p.cols[0], F.mid[0]) &&
         cover(b, 's', layout >= 2, a[2], a[3], &p.cols[1], F.mid[1]);
    ins(0, MB_ORM, 0, 0, 0), ins(1, MB_ANDM, 0, 1, 0);
  } else if (q.tmpl == 3) {
    p.ncols = 3;
    ok = cover(b, 'c', layout >= 1, a[0], a[1], &p.cols[0], F.mid[0]) &&
         cover(b, 's', layout >= 2, a[2], a[3], &p.cols[1], F.mid[1]);
    ins(0, MB_ORM, 0, 0, 0), ins(1, MB_ANDM, 0, 1, 0);
    if (a[4] == SSBDATE_920101) {  // date < max as NOT(date in [max, end)) (ssb/fixedlayout.cu:86-90)
      ok = ok && cover(b, 'd', layout >= 2, a[5], SSBDATE_990101, &p.cols[2], F.mid[2]);
      ins(2, MB_ORM, 1, 2, 0), ins(3, MB_NOT, 1, 1, 0), ins(4, MB_AND, 0, 1, 0);
    } else {
      ok = ok && cover(b, 'd', layout >= 2, a[4], a[5], &p.cols[2], F.mid[2]);
      ins(2, MB_ANDM, 0, 2, 0);
    }
  } else {
    p.ncols = 3;
    ok = cover(b, 'c', layout >= 1, a[0], a[1], &p.cols[0], F.mid[0]) &&
         cover(b, 's', layout >= 2, a[2], a[3], &p.cols[1], F.mid[1]) &&
         cover(b, 'm', layout >= 1, a[4], a[5], &p.cols[2], F.mid[2]);
    ins(0, MB_ORM, 0, 0, 0), ins(1, MB_ANDM, 0, 1, 0), ins(2, MB_ANDM, 0, 2, 0);
    if (a[7] < SSBDATE_990101 || a[6] > SSBDATE_920101) {
      p.ncols = 4;
      ok = ok && cover(b, 'd', false, a[6], a[7], &p.cols[3], F.mid[3]);
      ins(3, MB_ANDM, 0, 3, 0);
    }
  }
  return ok;
}

// The materialised plan (stages 1-3) of p into out / nq.
mb_status run_materialised(const mb_vprg &p, const mb_op &op, uint32_t ng, uint64_t n, int64_t *out, uint64_t *nq,
                           DevBufs &B, float *ms3) {
  const uint64_t W = mb_bitmap_stride(n);
  uint32_t *possi = (uint32_t *)B.get(W * 4), *unc = (uint32_t *)B.get(W * 4);
  uint32_t *rows = (uint32_t *)B.get((n + 1) * 4);
  uint64_t *cnt = (uint64_t *)B.get(8);
  if (!possi || !unc || !rows || !cnt) return fail(MB_ERR_OOM, "materialised plan scratch");
  const int chk = !mb_vprg_is_nochk(&p);
  Timer t;
  t.start();
  MB_CHECK(mb_vprg_eval(&p, chk, possi, chk ? unc : nullptr, nullptr, nullptr));
  if (ms3) ms3[0] = t.stop();
  t.start();
  MB_CHECK(mb_bitmap_to_rows(possi, chk ? unc : nullptr, n, rows, cnt, nullptr));
  if (ms3) ms3[1] = t.stop();
  t.start();
  MB_CHECK(mb_rows_grpby(rows, cnt, n + 1, &op, ng, out, nq, nullptr));
  if (ms3) ms3[2] = t.stop();
  return MB_OK;
}

// Per-query recipe bitmaps of ssb/controlled-demo.cu:19-96.
bool ssb_recipe(const ssb_schema *d, const mb_query &q, uint64_t n, mb_recipe &r, mb_instr *ins) {
  memset(&r, 0, sizeof(r));
  memset(ins, 0, sizeof(mb_instr) * MB_MAXNINSTR);
  r.factsz = n;
  const uint32_t *a = q.p;
  auto col = [&](int i, uint32_t nbit, uint32_t lo, uint32_t hi, const uint32_t *fk, const void *attr) {
    r.nbit[i] = nbit, r.min[i] = lo, r.max[i] = hi, r.dimsz[i] = 0xffffffffu, r.fk[i] = fk, r.attr[i] = attr;
  };
  auto in = [&](int i, uint32_t op, uint32_t s1) { ins[i].opcode = op, ins[i].dstreg = 0, ins[i].src1 = s1; };
  if (q.tmpl == 1) {
    col(0, 16, a[0], a[1], nullptr, d->loOrderDate);
    col(1, 8, a[2], a[3], nullptr, d->loDiscount);
    col(2, 8, a[4], a[5], nullptr, d->loQuantity);
    in(0, MB_ORM, 0), in(1, MB_ANDM, 1), in(2, MB_ANDM, 2);
  } else if (q.tmpl == 2) {
    col(0, 16, a[0], a[1], d->loPartKey, d->partMfgr);
    col(1, 8, a[2], a[3], nullptr, d->loSuppCity);
    in(0, MB_ORM, 0), in(1, MB_ANDM, 1);
  } else if (q.tmpl == 3) {
    col(0, 8, a[0], a[1], d->loCustKey, d->custCity);
    col(1, 8, a[2], a[3], nullptr, d->loSuppCity);
    col(2, 16, a[4], a[5], nullptr, d->loOrderDate);
    in(0, MB_ORM, 0), in(1, MB_ANDM, 1), in(2, MB_ANDM, 2);
  } else {
    col(0, 8, a[0], a[1], d->loCustKey, d->custCity);
    col(1, 8, a[2], a[3], nullptr, d->loSuppCity);
    col(2, 16, a[4], a[5], d->loPartKey, d->partMfgr);
    in(0, MB_ORM, 0), in(1, MB_ANDM, 1), in(2, MB_ANDM, 2);
    if (!(a[6] <= SSBDATE_920101 && a[7] >= SSBDATE_990101)) {
      col(3, 16, a[6], a[7], nullptr, d->loOrderDate);
      in(3, MB_ANDM, 3);
    }
  }
  return true;
}

// ------------------------------------------------------------ synth
mb_op synth_op(const synth_schema *d, uint64_t fa1lo, uint64_t fa1hi, uint64_t fa2lo, uint64_t fa2hi,
               uint64_t da1lo, uint64_t da1hi) {
  // _op (synth/synthdemo.cu:7-53): (a1 in R1 OR a2 in R2) AND dim.a1 in R3,
  // group by dim.a2, count; the key is not bound-checked
  mb_op o;
  memset(&o, 0, sizeof(o));
  const uint32_t w = d->bitwidth / 8;
  o.nsrc = 4;
  o.src[0] = src_of(d->factattr1, w);
  o.src[1] = src_of(d->factattr2, w);
  o.src[2] = src_of(d->dimattr1, 4, d->fkey);
  o.src[3] = src_of(d->dimattr2, 1, d->fkey);
  o.nclause = 2;
  o.clause_len[0] = 2, o.clause_len[1] = 1;
  o.terms[0].src = 0, o.terms[0].lo = fa1lo, o.terms[0].hi = fa1hi;
  o.terms[1].src = 1, o.terms[1].lo = fa2lo, o.terms[1].hi = fa2hi;
  o.terms[2].src = 2, o.terms[2].lo = da1lo, o.terms[2].hi = da1hi;
  o.nkey = 1;
  o.keys[0].src = 3, o.keys[0].xform = MB_X_ID, o.keys[0].div = 1, o.keys[0].base = 0, o.keys[0].mul = 1;
  o.vkind = MB_V_ONE;
  return o;
}

bool synth_recipe(const synth_schema *d, uint64_t n, uint32_t fa1lo, uint32_t fa1hi, uint32_t fa2lo, uint32_t fa2hi,
                  uint32_t da1lo, uint32_t da1hi, mb_recipe &r, mb_instr *ins) {
  memset(&r, 0, sizeof(r));
  memset(ins, 0, sizeof(mb_instr) * MB_MAXNINSTR);
  r.factsz = n;
  r.nbit[0] = r.nbit[1] = d->bitwidth, r.nbit[2] = 32;
  r.min[0] = fa1lo, r.max[0] = fa1hi, r.min[1] = fa2lo, r.max[1] = fa2hi, r.min[2] = da1lo, r.max[2] = da1hi;
  r.dimsz[0] = r.dimsz[1] = 0xffffffffu, r.dimsz[2] = (uint32_t)(n / 100);
  r.fk[2] = d->fkey;
  r.attr[0] = d->factattr1, r.attr[1] = d->factattr2, r.attr[2] = d->dimattr1;
  ins[0].opcode = MB_ORM, ins[0].src1 = 0;
  ins[1].opcode = MB_ORM, ins[1].src1 = 1;
  ins[2].opcode = MB_ANDM, ins[2].src1 = 2;
  return true;
}

bool same_u32(const uint32_t *a_dev, const uint32_t *b_host, size_t n, const char *what) {
  std::vector<uint32_t> h(n);
  cudaMemcpy(h.data(), a_dev, n * 4, cudaMemcpyDeviceToHost);
  for (size_t i = 0; i < n; ++i)
    if (h[i] != b_host[i]) {
      fprintf(stderr, "\n%s mismatch at %zu: expected %u, got %u", what, i, b_host[i], h[i]);
      return false;
    }
  return true;
}

}  // namespace
}  // namespace mb

using namespace mb;

// ============================================================ SSB
extern "C" size_t ssb_load(ssb_schema *host, ssb_schema *dev, const char *dir) {
  memset(host, 0, sizeof(*host));
  if (dev) memset(dev, 0, sizeof(*dev));
  size_t bytes = 0;
  if (!read_col(dir, "loCustKey", 0, (void **)&host->loCustKey, &bytes)) return 0;
  const size_t n = bytes / 4;
  size_t csz = 0, psz = 0;
  bool ok = read_col(dir, "loPartKey", n * 4, (void **)&host->loPartKey, nullptr) &&
            read_col(dir, "loOrderDate", n * 2, (void **)&host->loOrderDate, nullptr) &&
            read_col(dir, "loExtendedPrice", n * 4, (void **)&host->loExtendedPrice, nullptr) &&
            read_col(dir, "loRevenue", n * 4, (void **)&host->loRevenue, nullptr) &&
            read_col(dir, "loSupplyCost", n * 4, (void **)&host->loSupplyCost, nullptr) &&
            read_col(dir, "loSuppCity", n, (void **)&host->loSuppCity, nullptr) &&
            read_col(dir, "loQuantity", n, (void **)&host->loQuantity, nullptr) &&
            read_col(dir, "loDiscount", n, (void **)&host->loDiscount, nullptr) &&
            read_col(dir, "custCity", 0, (void **)&host->custCity, &csz) &&
            read_col(dir, "custMktSegment", csz, (void **)&host->custMktSegment, nullptr) &&
            read_col(dir, "partName", 0, (void **)&host->partName, &psz) &&
            read_col(dir, "partMfgr", psz, (void **)&host->partMfgr, nullptr) &&
            read_col(dir, "partColor", psz / 2, (void **)&host->partColor, nullptr) &&
            read_col(dir, "partType", psz / 2, (void **)&host->partType, nullptr) &&
            read_col(dir, "partSize", psz / 2, (void **)&host->partSize, nullptr) &&
            read_col(dir, "partContainer", psz / 2, (void **)&host->partContainer, nullptr);
  if (ok && dev) {
    struct {
      void **d;
      const void *h;
      size_t b;
    } cp[] = {{(void **)&dev->loCustKey, host->loCustKey, n * 4},
              {(void **)&dev->loPartKey, host->loPartKey, n * 4},
              {(void **)&dev->loOrderDate, host->loOrderDate, n * 2},
              {(void **)&dev->loExtendedPrice, host->loExtendedPrice, n * 4},
              {(void **)&dev->loRevenue, host->loRevenue, n * 4},
              {(void **)&dev->loSupplyCost, host->loSupplyCost, n * 4},
              {(void **)&dev->loSuppCity, host->loSuppCity, n},
              {(void **)&dev->loQuantity, host->loQuantity, n},
              {(void **)&dev->loDiscount, host->loDiscount, n},
              {(void **)&dev->custCity, host->custCity, csz},
              {(void **)&dev->custMktSegment, host->custMktSegment, csz},
              {(void **)&dev->partName, host->partName, psz},
              {(void **)&dev->partMfgr, host->partMfgr, psz},
              {(void **)&dev->partColor, host->partColor, psz / 2},
              {(void **)&dev->partType, host->partType, psz / 2},
              {(void **)&dev->partSize, host->partSize, psz / 2},
              {(void **)&dev->partContainer, host->partContainer, psz / 2}};
    for (auto &c : cp)
      if (ok && !(*c.d = to_dev(c.h, c.b))) {
        fprintf(stderr, "merle_b200: ssb_load: device allocation failed\n");
        ok = false;
      }
  }
  if (!ok) {
    ssb_free(host, dev);
    return 0;
  }
  return n;
}

extern "C" void ssb_free(ssb_schema *host, ssb_schema *dev) {
  for (ssb_schema *s : {host, dev}) {
    if (!s) continue;
    void **cols[] = {(void **)&s->loCustKey,      (void **)&s->loPartKey,  (void **)&s->loOrderDate,
                     (void **)&s->loExtendedPrice, (void **)&s->loRevenue, (void **)&s->loSupplyCost,
                     (void **)&s->loQuantity,     (void **)&s->loDiscount, (void **)&s->loSuppCity,
                     (void **)&s->custMktSegment, (void **)&s->custCity,   (void **)&s->partName,
                     (void **)&s->partMfgr,       (void **)&s->partColor,  (void **)&s->partType,
                     (void **)&s->partSize,       (void **)&s->partContainer};
    for (void **p : cols) {
      if (s == host) free(*p);
      else cudaFree(*p);
      *p = nullptr;
    }
  }
}

// One slab of ncol bins [bin[j], bin[j+1]) over a column (or a dimension
// attribute through a foreign key), the pointers into it in out[].
static float bmp_set(const mb_src &s, uint64_t n, const uint64_t *bin, uint32_t ncol, uint32_t **out) {
  const uint64_t stride = mb_bitmap_stride(n);
  uint32_t *slab = nullptr;
  for (uint32_t j = 0; j < ncol; ++j) out[j] = nullptr;
  if (cudaMalloc(&slab, stride * 4 * ncol) != cudaSuccess) {
    fprintf(stderr, "merle_b200: ssb_bmpcreate: device allocation failed\n");
    return 0;
  }
  Timer t;
  t.start();
  if (mb_bitmap_create(&s, n, bin, bin + 1, ncol, slab, stride, nullptr, nullptr) != MB_OK)
    fprintf(stderr, "merle_b200: ssb_bmpcreate: %s\n", mb_last_error());
  const float ms = t.stop();
  for (uint32_t j = 0; j < ncol; ++j) out[j] = slab + stride * j;
  return ms;
}

extern "C" void ssb_bmpcreate(const ssb_schema *host, const ssb_schema *dat, size_t n, ssb_bmp *o) {
  // dimension sizes from the largest keys (ssb/bmpidx-create.cu:122-131)
  uint32_t mp = 0, mc = 0;
  for (size_t i = 0; i < n; ++i) {
    if (host->loPartKey[i] > mp) mp = host->loPartKey[i];
    if (host->loCustKey[i] > mc) mc = host->loCustKey[i];
  }
  const uint64_t dp = (uint64_t)mp + 1, dc = (uint64_t)mc + 1;
  const mb_src date = src_of(dat->loOrderDate, 2), disc = src_of(dat->loDiscount, 1),
               qty = src_of(dat->loQuantity, 1), scity = src_of(dat->loSuppCity, 1),
               ccity = src_of(dat->custCity, 1, dat->loCustKey, dc),
               mfgr = src_of(dat->partMfgr, 2, dat->loPartKey, dp);
  const double mb = mb_bitmap_stride(n) * 4 / (1024.0 * 1024.0);
  printf("\nColumn\tMy(ms)\tWAH(ms)\tMy(MB)\tWAH(MB)\n");
  struct {
    const char *name;
    const mb_src &s;
    const uint64_t *bin;
    uint32_t ncol;
    uint32_t **out;
  } sets[] = {{"loOrderDate_Sparse", date, dateSpBin, 7, o->dateSparse},
              {"loDiscount_Sparse", disc, discntSpBin, 4, o->discntSparse},
              {"loQuantity_Sparse", qty, qtySpBin, 5, o->qtySparse},
              {"loSuppCity_Sparse", scity, sCitySpBin, 5, o->sCitySparse},
              {"custCity_Sparse", ccity, sCitySpBin, 5, o->cCitySparse},
              {"partMfgr_Sparse", mfgr, mfgrSpBin, 5, o->mfgrSparse},
              {"loOrderDate_Dense", date, dateDeBin, 4, o->dateDense},
              {"loDiscount_Dense", disc, discntDeBin, 11, o->discntDense},
              {"loQuantity_Dense", qty, qtyDeBin, 10, o->qtyDense},
              {"loSuppCity_Dense", scity, sCityDeBin, 3, o->sCityDense},
              {"custCity_Dense", ccity, sCityDeBin, 3, o->cCityDense},
              {"partMfgr_Dense", mfgr, mfgrDeBin, 5, o->mfgrDense}};
  double total = 0;
  for (auto &s : sets) {
    const float ms = bmp_set(s.s, n, s.bin, s.ncol, s.out);
    total += ms;
    printf("%s\t%.2f\t0.00\t%.2f\t0.00\n", s.name, ms, mb * s.ncol);
  }
  printf("Total\t%.2f\t0.00\t-\t-\n", total);
}

extern "C" void ssb_bmpfree(ssb_bmp *o) {
  uint32_t **firsts[] = {o->dateSparse,  o->dateDense,  o->discntSparse, o->discntDense,
                         o->qtySparse,   o->qtyDense,   o->mfgrSparse,   o->mfgrDense,
                         o->sCitySparse, o->sCityDense, o->cCitySparse,  o->cCityDense};
  for (uint32_t **f : firsts) cudaFree(f[0]), f[0] = nullptr;
}

extern "C" uint32_t *ssb_cpujoin(const ssb_schema *dat, size_t n) {
  // The reference computes these on the host (ssb/cpuref.c:244-299); this
  // library has no CPU path: the table goes to an engine and each query runs
  // there (rule plan over the engine's own index).
  uint32_t *res = (uint32_t *)calloc(SUMGRP_ALL + 1, sizeof(uint32_t));
  if (!res) return nullptr;
  uint32_t mp = 0, mc = 0;
  for (size_t i = 0; i < n; ++i) {
    if (dat->loPartKey[i] > mp) mp = dat->loPartKey[i];
    if (dat->loCustKey[i] > mc) mc = dat->loCustKey[i];
  }
  mb_engine *e = nullptr;
  mb_star_host h;
  memset(&h, 0, sizeof(h));
  h.nrows = n, h.ncust = (uint64_t)mc + 1, h.nsupp = 0, h.npart = (uint64_t)mp + 1;
  h.custkey = dat->loCustKey, h.partkey = dat->loPartKey, h.orderdate = dat->loOrderDate;
  h.extendedprice = dat->loExtendedPrice, h.revenue = dat->loRevenue, h.supplycost = dat->loSupplyCost;
  h.quantity = dat->loQuantity, h.discount = dat->loDiscount, h.suppcity = dat->loSuppCity;
  h.custcity = dat->custCity, h.partmfgr = dat->partMfgr;
  std::vector<int64_t> out(1024);
  bool ok = mb_engine_create(0, &e) == MB_OK && mb_engine_load_star(e, &h) == MB_OK && mb_engine_build_index(e) == MB_OK;
  for (int i = 0; ok && i < 13; ++i) {
    ok = mb_engine_query(e, &SSB13[i].q, nullptr, out.data(), nullptr, nullptr) == MB_OK;
    const uint32_t off = ssb_offset(i), ng = query_ngroups(SSB13[i].q);
    for (uint32_t g = 0; ok && g < ng; ++g) res[off + g] = (uint32_t)(uint64_t)out[g];
  }
  if (!ok) fprintf(stderr, "merle_b200: ssb_cpujoin: %s\n", mb_last_error());
  mb_engine_destroy(e);
  if (!ok) {
    free(res);
    return nullptr;
  }
  return res;
}

extern "C" uint32_t *ssb_bmp_fixed(const ssb_schema *dat, ssb_bmp *bmp, size_t n) {
  uint32_t *res = nullptr;
  if (cudaMalloc(&res, (size_t)SUMGRP_ALL * 5 * 4) != cudaSuccess) {
    fprintf(stderr, "merle_b200: ssb_bmp_fixed: device allocation failed\n");
    return nullptr;
  }
  cudaMemset(res, 0, (size_t)SUMGRP_ALL * 5 * 4);
  DevBufs B;
  int64_t *out = (int64_t *)B.get(1024 * 8);
  uint64_t *nq = (uint64_t *)B.get(8);
  const SsbSrc S = ssb_srcs(dat);
  const char *lay[3] = {"Sparse", "Medium", "Dense"};
  printf("\nCase\tBinType\tJoin\tOurs\tDirect\tNoFuse\tTMA");
  bool ok = out && nq;
  for (int i = 0; ok && i < 13; ++i) {
    const mb_query &q = SSB13[i].q;
    const uint32_t ng = query_ngroups(q), off = ssb_offset(i);
    mb_op op;
    ssb_build_op(S, q, op);
    for (int l = 0; ok && l < 3; ++l) {
      FixedPrg F;
      if (!fixed_prg(bmp, q, n, l, F)) {
        fprintf(stderr, "\nmerle_b200: ssb_bmp_fixed: %s: %s", SSB13[i].name, mb_last_error());
        ok = false;
        break;
      }
      Timer t;
      float tj = 0, tf, td, tm[3] = {0, 0, 0}, tt;
      if (l == 0) {
        t.start();
        ok = ok && mb_join_grpby(n, &op, ng, out, nq, nullptr) == MB_OK;
        tj = t.stop();
        trunc32(out, res + off, ng);
      }
      t.start();
      ok = ok && mb_vprg_grpby(&F.p, &op, ng, out, nq, nullptr, nullptr) == MB_OK;
      tf = t.stop();
      if (l == 2) trunc32(out, res + SUMGRP_ALL + off, ng);
      mb_launch direct;
      memset(&direct, 0, sizeof(direct));
      direct.staging = MB_STAGE_DIRECT, direct.grp_strategy = MB_GRP_GLOBAL;
      t.start();
      ok = ok && mb_vprg_grpby(&F.p, &op, ng, out, nq, &direct, nullptr) == MB_OK;
      td = t.stop();
      if (l == 2) trunc32(out, res + 2 * SUMGRP_ALL + off, ng);
      ok = ok && run_materialised(F.p, op, ng, n, out, nq, B, tm) == MB_OK;
      if (l == 2) trunc32(out, res + 3 * SUMGRP_ALL + off, ng);
      mb_launch tma;
      memset(&tma, 0, sizeof(tma));
      tma.staging = MB_STAGE_TMA;
      t.start();
      ok = ok && mb_vprg_grpby(&F.p, &op, ng, out, nq, &tma, nullptr) == MB_OK;
      tt = t.stop();
      if (l == 0) trunc32(out, res + 4 * SUMGRP_ALL + off, ng);
      printf("\n%s\t%s\t%.4f\t%.4f\t%.4f\t%.4f\t%.4f", SSB13[i].name, lay[l], tj, tf, td, tm[0] + tm[1] + tm[2], tt);
    }
  }
  printf("\n");
  cudaDeviceSynchronize();
  if (!ok) {
    fprintf(stderr, "merle_b200: ssb_bmp_fixed: %s\n", mb_last_error());
    cudaFree(res);
    return nullptr;
  }
  return res;
}

// The 13 queries over recipe bitmaps; slots: 1 << (kind + 1) set in `which`
// for perfect / many_or / candchk into res + (kind + 1) * SUMGRP_ALL, bit 0
// the join into res, bit 4 the materialised plan of the perfect recipe into
// res + matslot * SUMGRP_ALL.
static uint32_t *ssb_control(const ssb_schema *dat, size_t n, uint32_t slots, uint32_t which, int matslot,
                             const char *who) {
  uint32_t *res = nullptr;
  if (cudaMalloc(&res, (size_t)SUMGRP_ALL * slots * 4) != cudaSuccess) {
    fprintf(stderr, "merle_b200: %s: device allocation failed\n", who);
    return nullptr;
  }
  cudaMemset(res, 0, (size_t)SUMGRP_ALL * slots * 4);
  DevBufs B;
  int64_t *out = (int64_t *)B.get(1024 * 8);
  uint64_t *nq = (uint64_t *)B.get(8);
  const SsbSrc S = ssb_srcs(dat);
  const char *kinds[3] = {"Perfect", "AllAlig", "MisAlig"};
  bool ok = out && nq;
  for (int i = 0; ok && i < 13; ++i) {
    const mb_query &q = SSB13[i].q;
    const uint32_t ng = query_ngroups(q), off = ssb_offset(i);
    mb_op op;
    ssb_build_op(S, q, op);
    if (which & 1u) {
      ok = mb_join_grpby(n, &op, ng, out, nq, nullptr) == MB_OK;
      trunc32(out, res + off, ng);
    }
    for (int k = 0; ok && k < 3; ++k) {
      const bool fused = (which >> (k + 1)) & 1u, mat = k == 0 && ((which >> 4) & 1u);
      if (!fused && !mat) continue;
      mb_recipe r;
      mb_instr ins[MB_MAXNINSTR];
      ssb_recipe(dat, q, n, r, ins);
      mb_owned_vprg P;
      ok = mb_recipe_build(&r, k, ins, &P, nullptr) == MB_OK;
      if (!ok) break;
      Timer t;
      float tf = 0, tm[3] = {0, 0, 0};
      if (fused) {
        t.start();
        ok = mb_vprg_grpby(&P.prg, &op, ng, out, nq, nullptr, nullptr) == MB_OK;
        tf = t.stop();
        trunc32(out, res + (k + 1) * SUMGRP_ALL + off, ng);
      }
      if (ok && mat) {
        ok = run_materialised(P.prg, op, ng, n, out, nq, B, tm) == MB_OK;
        trunc32(out, res + matslot * SUMGRP_ALL + off, ng);
      }
      cudaDeviceSynchronize();
      mb_owned_vprg_release(&P);
      printf("\n%s\t%s\t0\t%.4f\t%.4f\t%.4f\t%.4f", SSB13[i].name, kinds[k], tf, tm[0], tm[1], tm[2]);
    }
  }
  printf("\n");
  cudaDeviceSynchronize();
  if (!ok) {
    fprintf(stderr, "merle_b200: %s: %s\n", who, mb_last_error());
    cudaFree(res);
    return nullptr;
  }
  return res;
}

extern "C" uint32_t *ssb_bmp_control(const ssb_schema *dat, size_t n) {
  return ssb_control(dat, n, 4, 0x0fu, 0, "ssb_bmp_control");
}
extern "C" uint32_t *ssb_bmp_control_abl_fuse(const ssb_schema *dat, size_t n) {
  uint32_t *r = ssb_control(dat, n, 2, 0x02u, 0, "ssb_bmp_control_abl_fuse");
  if (r) cudaMemcpy(r, r + SUMGRP_ALL, SUMGRP_ALL * 4, cudaMemcpyDeviceToDevice);
  return r;
}
extern "C" uint32_t *ssb_bmp_control_abl_nofuse(const ssb_schema *dat, size_t n) {
  return ssb_control(dat, n, 1, 0x10u, 0, "ssb_bmp_control_abl_nofuse");
}

// ------------------------------------------------------- WAH baseline
// The reference's compressed-bitmap baseline (ssb/wah-demo.cu:22-240,
// synth/wah_roast.cu:5-36) on this library's WAH kernels: one bitmap per
// predicate, compressed with row 31g + j at bit 30 - j (dbjoinFlatWah's
// order); timed: WAH_REPS repetitions of the streams' AND chain and the
// decompression of the result (the synthetic query: OR, then AND), with
// events around them, in milliseconds per repetition.
namespace {
constexpr int WAH_REPS = 100;

struct WahPred {
  mb_src src;
  uint64_t lo, hi;
};

bool wah_streams(const std::vector<WahPred> &preds, uint64_t n, DevBufs &B, std::vector<uint32_t *> &w,
                 std::vector<uint64_t> &wn, uint32_t **bm) {
  const uint64_t G = mb_wah_groups(n), stride = mb_bitmap_stride(n);
  *bm = static_cast<uint32_t *>(B.get(stride * 4));
  if (!*bm) return false;
  for (const WahPred &p : preds) {
    uint32_t *s = static_cast<uint32_t *>(B.get(G * 4));
    uint64_t k = 0;
    if (!s || mb_bitmap_create(&p.src, n, &p.lo, &p.hi, 1, *bm, stride, nullptr, nullptr) != MB_OK ||
        mb_wah_encode(*bm, n, MB_WAH_MSB, s, G, &k, nullptr) != MB_OK)
      return false;
    w.push_back(s);
    wn.push_back(k);
  }
  return true;
}

// ops[i] combines the running result with stream i + 1; decode: expand the
// result each repetition.
bool wah_time(const std::vector<uint32_t *> &w, const std::vector<uint64_t> &wn, const std::vector<uint32_t> &ops,
              bool decode, uint64_t n, uint32_t *bm, DevBufs &B, float *ms) {
  const uint64_t G = mb_wah_groups(n);
  uint32_t *t[2] = {static_cast<uint32_t *>(B.get(G * 4)), static_cast<uint32_t *>(B.get(G * 4))};
  if (!t[0] || !t[1]) return false;
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess) return false;
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    return false;
  }
  bool ok = cudaEventRecord(e0) == cudaSuccess;
  for (int rep = 0; ok && rep < WAH_REPS; ++rep) {
    const uint32_t *r = w[0];
    uint64_t rn = wn[0];
    for (size_t k = 1; ok && k < w.size(); ++k) {
      uint32_t *o = t[k & 1];
      uint64_t on = 0;
      ok = mb_wah_op(ops[k - 1], r, rn, w[k], wn[k], G, o, G, &on, nullptr) == MB_OK;
      r = o, rn = on;
    }
    if (ok && decode) ok = mb_wah_decode(r, rn, MB_WAH_MSB, n, bm, nullptr) == MB_OK;
  }
  ok = ok && cudaEventRecord(e1) == cudaSuccess && cudaEventSynchronize(e1) == cudaSuccess &&
       cudaEventElapsedTime(ms, e0, e1) == cudaSuccess;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *ms /= WAH_REPS;
  return ok;
}
}  // namespace

extern "C" void ssb_wah(const ssb_schema *, const ssb_schema *dat, size_t factSz) {
  const SsbSrc S = ssb_srcs(dat);
  puts("\nCase\tWAH\tRTScan");
  for (const SsbQ &sq : SSB13) {
    const uint32_t *p = sq.q.p;
    std::vector<WahPred> preds;
    switch (sq.q.tmpl) {
    case 1: preds = {{S.date, p[0], p[1]}, {S.disc, p[2], p[3]}, {S.qty, p[4], p[5]}}; break;
    case 2: preds = {{S.mfgr, p[0], p[1]}, {S.scity, p[2], p[3]}}; break;
    case 3: preds = {{S.ccity, p[0], p[1]}, {S.scity, p[2], p[3]}, {S.date, p[4], p[5]}}; break;
    default: preds = {{S.ccity, p[0], p[1]}, {S.scity, p[2], p[3]}, {S.mfgr, p[4], p[5]}, {S.date, p[6], p[7]}};
    }
    DevBufs B;
    std::vector<uint32_t *> w;
    std::vector<uint64_t> wn;
    uint32_t *bm = nullptr;
    float ms = 0;
    const std::vector<uint32_t> ands(preds.size() - 1, MB_WAH_AND);
    if (!wah_streams(preds, factSz, B, w, wn, &bm) || !wah_time(w, wn, ands, true, factSz, bm, B, &ms))
      printf("%s\tfailed: %s\n", sq.name, mb_last_error());
    else  // RTScan (an OptiX ray-tracing scan) is not run here
      printf("%s\t%.4f\tunavailable\n", sq.name, ms);
  }
}

extern "C" bool ssb_demoall(const char *dir) {
  ssb_schema host, dev;
  const size_t n = ssb_load(&host, &dev, dir);
  if (n == 0) return false;
  ssb_wah(&host, &dev, n);
  uint32_t *want = ssb_cpujoin(&host, n);
  bool ok = want != nullptr;
  ssb_bmp bmp;
  memset(&bmp, 0, sizeof(bmp));
  if (ok) ssb_bmpcreate(&host, &dev, n, &bmp);
  uint32_t *r = ok ? ssb_bmp_fixed(&dev, &bmp, n) : nullptr;
  ok = ok && r;
  const char *fixed[5] = {"Join", "Our fixed-layout", "Direct loads", "No fusion", "TMA staged"};
  for (int s = 0; ok && s < 5; ++s) ok = same_u32(r + s * SUMGRP_ALL, want, SUMGRP_ALL, fixed[s]);
  cudaFree(r);
  ssb_bmpfree(&bmp);
  r = ok ? ssb_bmp_control(&dev, n) : nullptr;
  ok = ok && r;
  const char *ctl[4] = {"Controlled join", "Our controlled-layout", "Controlled aligned", "Controlled misaligned"};
  for (int s = 0; ok && s < 4; ++s) ok = same_u32(r + s * SUMGRP_ALL, want, SUMGRP_ALL, ctl[s]);
  cudaFree(r);
  free(want);
  ssb_free(&host, &dev);
  return ok;
}

// ============================================================ synth
extern "C" size_t synth_load(synth_schema *host, synth_schema *dev, const char *dir) {
  memset(host, 0, sizeof(*host));
  if (dev) memset(dev, 0, sizeof(*dev));
  size_t fkb = 0, ab = 0;
  bool ok = read_col(dir, "fk", 0, (void **)&host->fkey, &fkb) && read_col(dir, "a1", 0, &host->factattr1, &ab) &&
            read_col(dir, "a2", ab, &host->factattr2, nullptr);
  const size_t n = fkb / 4;
  ok = ok && n > 0 && (ab * 8) % n == 0;
  if (ok) {
    host->bitwidth = (uint32_t)(ab * 8 / n);
    ok = host->bitwidth == 8 || host->bitwidth == 16 || host->bitwidth == 32 || host->bitwidth == 64;
  }
  // the dimension (synth/cpuref.c:75-86): attr1 = key, attr2 = the C
  // library's rand() after srand(13458786), 8 bits
  const size_t dimsz = n / 100;
  if (ok) {
    host->dimattr1 = (uint32_t *)malloc((dimsz ? dimsz : 1) * 4);
    host->dimattr2 = (uint8_t *)malloc(dimsz ? dimsz : 1);
    ok = host->dimattr1 && host->dimattr2;
  }
  if (ok) {
    srand(13458786);
    for (size_t i = 0; i < dimsz; ++i) host->dimattr1[i] = (uint32_t)i, host->dimattr2[i] = (uint8_t)rand();
  }
  if (ok && dev) {
    dev->bitwidth = host->bitwidth;
    ok = (dev->fkey = (uint32_t *)to_dev(host->fkey, fkb)) && (dev->factattr1 = to_dev(host->factattr1, ab)) &&
         (dev->factattr2 = to_dev(host->factattr2, ab)) &&
         (dev->dimattr1 = (uint32_t *)to_dev(host->dimattr1, dimsz * 4)) &&
         (dev->dimattr2 = (uint8_t *)to_dev(host->dimattr2, dimsz));
  }
  if (!ok) {
    fprintf(stderr, "merle_b200: synth_load: cannot load %s\n", dir);
    synth_free(host, dev);
    return 0;
  }
  return n;
}

extern "C" void synth_free(synth_schema *host, synth_schema *dev) {
  if (host) {
    free(host->factattr1), free(host->factattr2), free(host->fkey), free(host->dimattr1), free(host->dimattr2);
    host->factattr1 = host->factattr2 = nullptr, host->fkey = host->dimattr1 = nullptr, host->dimattr2 = nullptr;
  }
  if (dev) {
    cudaFree(dev->factattr1), cudaFree(dev->factattr2), cudaFree(dev->fkey), cudaFree(dev->dimattr1),
        cudaFree(dev->dimattr2);
    dev->factattr1 = dev->factattr2 = nullptr, dev->fkey = dev->dimattr1 = nullptr, dev->dimattr2 = nullptr;
  }
}

extern "C" void synth_join(const synth_schema *dat, size_t n, uint64_t fa1lo, uint64_t fa1hi, uint64_t fa2lo,
                           uint64_t fa2hi, uint64_t da1lo, uint64_t da1hi, uint32_t *grpout) {
  DevBufs B;
  int64_t *out = (int64_t *)B.get(256 * 8);
  uint64_t *nq = (uint64_t *)B.get(8);
  const mb_op op = synth_op(dat, fa1lo, fa1hi, fa2lo, fa2hi, da1lo, da1hi);
  if (!out || !nq || mb_join_grpby(n, &op, 256, out, nq, nullptr) != MB_OK) {
    fprintf(stderr, "merle_b200: synth_join: %s\n", mb_last_error());
    return;
  }
  trunc32(out, grpout, 256);
}

extern "C" void synth_ref(const synth_schema *host, size_t n, uint64_t fa1lo, uint64_t fa1hi, uint64_t fa2lo,
                          uint64_t fa2hi, uint64_t da1lo, uint64_t da1hi, uint32_t *grpout) {
  // The reference computes this on the host (synth/cpuref.c:123-163); this
  // library has no CPU path: the columns go to the device for the join.
  memset(grpout, 0, 256 * 4);
  const size_t w = host->bitwidth / 8, dimsz = n / 100;
  synth_schema d;
  d.bitwidth = host->bitwidth;
  d.factattr1 = to_dev(host->factattr1, n * w);
  d.factattr2 = to_dev(host->factattr2, n * w);
  d.fkey = (uint32_t *)to_dev(host->fkey, n * 4);
  d.dimattr1 = (uint32_t *)to_dev(host->dimattr1, dimsz * 4);
  d.dimattr2 = (uint8_t *)to_dev(host->dimattr2, dimsz);
  uint32_t *g = nullptr;
  if (d.factattr1 && d.factattr2 && d.fkey && d.dimattr1 && d.dimattr2 && cudaMalloc(&g, 256 * 4) == cudaSuccess) {
    synth_join(&d, n, fa1lo, fa1hi, fa2lo, fa2hi, da1lo, da1hi, g);
    cudaMemcpy(grpout, g, 256 * 4, cudaMemcpyDeviceToHost);
  } else {
    fprintf(stderr, "merle_b200: synth_ref: device allocation failed\n");
  }
  cudaFree(g);
  synth_free(nullptr, &d);
}

extern "C" float4 synth_bmp(const synth_schema *dat, uint32_t n, uint32_t fa1lo, uint32_t fa1hi, uint32_t fa2lo,
                            uint32_t fa2hi, uint32_t da1lo, uint32_t da1hi, uint32_t *grpout, int ty) {
  float4 r = make_float4(0, 0, 0, 0);
  DevBufs B;
  int64_t *out = (int64_t *)B.get(256 * 8);
  uint64_t *nq = (uint64_t *)B.get(8);
  const mb_op op = synth_op(dat, fa1lo, fa1hi, fa2lo, fa2hi, da1lo, da1hi);
  Timer t;
  if (!out || !nq) return r;
  if (ty < 0) {
    t.start();
    const mb_status s = mb_join_grpby(n, &op, 256, out, nq, nullptr);
    r.x = t.stop();
    if (s != MB_OK) fprintf(stderr, "merle_b200: synth_bmp: %s\n", mb_last_error());
    trunc32(out, grpout, 256);
    return r;
  }
  mb_recipe rc;
  mb_instr ins[MB_MAXNINSTR];
  synth_recipe(dat, n, fa1lo, fa1hi, fa2lo, fa2hi, da1lo, da1hi, rc, ins);
  mb_owned_vprg P;
  if (mb_recipe_build(&rc, ty % 3, ins, &P, nullptr) != MB_OK) {
    fprintf(stderr, "merle_b200: synth_bmp: %s\n", mb_last_error());
    return r;
  }
  mb_status s = MB_OK;
  if (ty < 3) {
    t.start();
    s = mb_vprg_grpby(&P.prg, &op, 256, out, nq, nullptr, nullptr);
    r.x = t.stop();
  } else {
    float tm[3] = {0, 0, 0};
    s = run_materialised(P.prg, op, 256, n, out, nq, B, tm);
    r.x = tm[0], r.y = tm[1], r.z = tm[2];
  }
  if (s != MB_OK) fprintf(stderr, "merle_b200: synth_bmp: %s\n", mb_last_error());
  trunc32(out, grpout, 256);
  cudaDeviceSynchronize();
  mb_owned_vprg_release(&P);
  return r;
}

extern "C" float2 synth_method(const synth_schema *dat, uint32_t n, uint32_t fa1lo, uint32_t fa1hi, uint32_t fa2lo,
                               uint32_t fa2hi, uint32_t da1lo, uint32_t da1hi) {
  float2 r = make_float2(0, 0);
  DevBufs B;
  int64_t *out = (int64_t *)B.get(512 * 8);
  uint64_t *nq = (uint64_t *)B.get(16);
  const mb_op op = synth_op(dat, fa1lo, fa1hi, fa2lo, fa2hi, da1lo, da1hi);
  mb_recipe rc;
  mb_instr ins[MB_MAXNINSTR];
  synth_recipe(dat, n, fa1lo, fa1hi, fa2lo, fa2hi, da1lo, da1hi, rc, ins);
  mb_owned_vprg P;
  if (!out || !nq || mb_recipe_build(&rc, MB_RECIPE_PERFECT, ins, &P, nullptr) != MB_OK) {
    fprintf(stderr, "merle_b200: synth_method: %s\n", mb_last_error());
    return r;
  }
  mb_launch l1, l4;
  memset(&l1, 0, sizeof(l1));
  memset(&l4, 0, sizeof(l4));
  l1.words_per_lane = 1, l4.words_per_lane = 4;
  Timer t;
  t.start();
  mb_status s = mb_vprg_grpby(&P.prg, &op, 256, out, nq, &l1, nullptr);
  r.x = t.stop();
  t.start();
  if (s == MB_OK) s = mb_vprg_grpby(&P.prg, &op, 256, out + 256, nq + 1, &l4, nullptr);
  r.y = t.stop();
  std::vector<int64_t> h(512);
  cudaMemcpy(h.data(), out, 512 * 8, cudaMemcpyDeviceToHost);
  if (s != MB_OK) fprintf(stderr, "merle_b200: synth_method: %s\n", mb_last_error());
  for (int i = 0; s == MB_OK && i < 256; ++i)
    if (h[i] != h[i + 256]) {
      fprintf(stderr, "merle_b200: synth_method: tile widths disagree at %d: %lld != %lld\n", i, (long long)h[i],
              (long long)h[i + 256]);
      break;
    }
  mb_owned_vprg_release(&P);
  return r;
}

extern "C" void synth_wah(const synth_schema *dat, uint32_t factsz, uint32_t fa1lo, uint32_t fa1hi, uint32_t fa2lo,
                          uint32_t fa2hi, uint32_t da1lo, uint32_t da1hi) {
  // (a1 in R1 OR a2 in R2) AND key in R3: the dimension attribute is the key
  // itself (synth/cpuref.c:80), so its predicate is a range on the key column
  const uint32_t w = dat->bitwidth / 8;
  const std::vector<WahPred> preds = {{src_of(dat->factattr1, w), fa1lo, fa1hi},
                                      {src_of(dat->factattr2, w), fa2lo, fa2hi},
                                      {src_of(dat->fkey, 4), da1lo, da1hi}};
  DevBufs B;
  std::vector<uint32_t *> ws;
  std::vector<uint64_t> wn;
  uint32_t *bm = nullptr;
  float ms = 0;
  if (!wah_streams(preds, factsz, B, ws, wn, &bm) ||
      !wah_time(ws, wn, {MB_WAH_OR, MB_WAH_AND}, false, factsz, bm, B, &ms))
    printf("\tfailed: %s\n", mb_last_error());
  else
    printf("\t%.4f\n", ms);
}

extern "C" double *window_zipf(double s, size_t n, size_t win) {
  // Zipf(s) over values 1, 2, ...: P(k) = k^-s / zeta(s), with zeta(s) from
  // the alternating (Dirichlet eta) series over its first 50,000 terms,
  // zeta(s) = eta(s) / (1 - 2^(1-s)); window x sums P(k) for k in
  // [x + 1, x + win], values above 100,000 left out (synth/window_zipf.c).
  if (!(s > 1.0)) return nullptr;
  double *p = (double *)malloc((n ? n : 1) * sizeof(double));
  if (!p) return nullptr;
  double eta = 0, sg = 1;
  for (int k = 1; k <= 50000; ++k, sg = -sg) eta += sg / pow((double)k, s);
  const double zeta = eta / (1.0 - pow(2.0, 1.0 - s));
  const size_t kmax = n + win < 100000 ? n + win : 100000;
  std::vector<double> inv(kmax + 1, 0.0);
  for (size_t k = 1; k <= kmax; ++k) inv[k] = 1.0 / pow((double)k, s);
  for (size_t x = 0; x < n; ++x) {
    double acc = 0;
    for (size_t k = x + 1; k < x + win + 1 && k <= kmax; ++k) acc += inv[k];
    p[x] = acc / zeta;
  }
  return p;
}

extern "C" bool synth_demoall(const char *dir) {
  // the cases, skews and selectivity ladders of synth/cpuref.c:188-196
  static const char *cases[] = {"04_16", "04_32", "08_16", "08_32", "12_16",
                                "12_32", "16_16", "16_32", "20_16", "20_32"};
  static const double skews[] = {1.04, 1.04, 1.08, 1.08, 1.12, 1.12, 1.16, 1.16, 1.2, 1.2};
  static const double colsel[11] = {.02, .04, .06, .09, .12, .18, .25, .39, .51, .67, .82};
  static const double fulsel[11] = {1 / 512.0, 1 / 256.0, 1 / 128.0, 1 / 64.0, 1 / 32.0, 1 / 16.0,
                                    1 / 8.0,   1 / 4.0,   .4,        .6,        .8};
  char path[1024];
  synth_schema host, dev;
  puts("\n\nSeletiv\tMethod1\tMethod2");
  snprintf(path, sizeof(path), "%s/%s", dir, cases[1]);
  size_t n = synth_load(&host, &dev, path);
  if (n == 0) return false;
  double *win = window_zipf(skews[1], 1024, 60);
  for (int i = 0; i < 7 && win; ++i) {
    uint32_t lo = 0, hi = 60;
    while (lo < 1023 && win[lo] > colsel[i]) ++lo, ++hi;
    const float2 t = synth_method(&dev, (uint32_t)n, lo, hi, lo, hi, lo, hi);
    printf("%.5f\t%.4f\t%.4f\n", fulsel[i], t.x, t.y);
  }
  free(win);
  synth_free(&host, &dev);
  puts("\nSkew\tBitW\tSeletiv\tJoin\tPerfect\tManyOrs\tCandChk\tPftStg1\tPftStg2\tPftStg3"
       "\tOrsStg1\tOrsStg2\tOrsStg3\tChkStg1\tChkStg2\tChkStg3\tWAH");
  bool ok = true;
  for (int c = 0; ok && c < 10; ++c) {
    snprintf(path, sizeof(path), "%s/%s", dir, cases[c]);
    n = synth_load(&host, &dev, path);
    if (n == 0) return false;
    win = window_zipf(skews[c], 1024, 60);
    uint32_t *g = nullptr;
    ok = win && cudaMalloc(&g, 256 * 4) == cudaSuccess;
    for (int o = 1; ok && o < 11; ++o) {
      uint32_t lo = 0, hi = 60;
      while (lo < 1023 && win[lo] > colsel[o]) ++lo, ++hi;
      printf("%.2f\t%s\t%.5f", skews[c], cases[c] + 3, fulsel[o]);
      uint32_t want[256];
      synth_ref(&host, n, lo, hi, lo, hi, lo, hi, want);
      for (int ty = -1; ok && ty < 6; ++ty) {
        const float4 t = synth_bmp(&dev, (uint32_t)n, lo, hi, lo, hi, lo, hi, g, ty);
        if (ty >= 3) printf("\t%.4f\t%.4f\t%.4f", t.x, t.y, t.z);
        else printf("\t%.4f", t.x);
        ok = same_u32(g, want, 256, "synth");
      }
      if (host.bitwidth == 32) synth_wah(&dev, (uint32_t)n, lo, hi, lo, hi, lo, hi);
      else puts("\t0.0");
    }
    cudaFree(g);
    free(win);
    synth_free(&host, &dev);
  }
  return ok;
}
