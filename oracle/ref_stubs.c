/*
 * ref_stubs.c - link stubs for oracle/_ref/libcpuref.so.  TEST INFRASTRUCTURE.
 *
 * The reference's CPU oracle files (ssb/cpuref.c, synth/cpuref.c) also hold the
 * reference's benchmark drivers (ssb_demoall, synth_demoall), which call GPU
 * benchmark functions defined in .cu files that the CPU oracle library does not
 * compile.  These stubs only satisfy the dynamic linker; the tests call the
 * oracle functions (s1ref..s4ref, ssb_cpujoin, synth_ref, window_zipf) and
 * never the drivers.  Each stub reports the misuse and returns an empty result.
 */
#include <stdio.h>
#include <stdint.h>
#include <stddef.h>

struct ssb_schema;
struct ssb_bmp;
struct synth_schema;
typedef struct { float x, y; } stub_float2;
typedef struct { float x, y, z, w; } stub_float4;

static void misuse(const char *f) { fprintf(stderr, "oracle/_ref: %s is not built into the CPU oracle\n", f); }

void ssb_wah(const struct ssb_schema *h, const struct ssb_schema *d, size_t n) { (void)h; (void)d; (void)n; misuse("ssb_wah"); }
void ssb_bmpcreate(const struct ssb_schema *h, const struct ssb_schema *d, size_t n, struct ssb_bmp *o) { (void)h; (void)d; (void)n; (void)o; misuse("ssb_bmpcreate"); }
void ssb_bmpfree(struct ssb_bmp *o) { (void)o; misuse("ssb_bmpfree"); }
uint32_t *ssb_bmp_fixed(const struct ssb_schema *d, struct ssb_bmp *b, size_t n) { (void)d; (void)b; (void)n; misuse("ssb_bmp_fixed"); return NULL; }
uint32_t *ssb_bmp_control(const struct ssb_schema *d, size_t n) { (void)d; (void)n; misuse("ssb_bmp_control"); return NULL; }
stub_float2 synth_method(const struct synth_schema *d, uint32_t n, uint32_t a, uint32_t b, uint32_t c, uint32_t e, uint32_t f, uint32_t g) {
  (void)d; (void)n; (void)a; (void)b; (void)c; (void)e; (void)f; (void)g; misuse("synth_method"); stub_float2 r = {0, 0}; return r;
}
stub_float4 synth_bmp(const struct synth_schema *d, uint32_t n, uint32_t a, uint32_t b, uint32_t c, uint32_t e, uint32_t f, uint32_t g, uint32_t *o, int ty) {
  (void)d; (void)n; (void)a; (void)b; (void)c; (void)e; (void)f; (void)g; (void)o; (void)ty; misuse("synth_bmp"); stub_float4 r = {0, 0, 0, 0}; return r;
}
void synth_wah(const struct synth_schema *d, uint32_t n, uint32_t a, uint32_t b, uint32_t c, uint32_t e, uint32_t f, uint32_t g) {
  (void)d; (void)n; (void)a; (void)b; (void)c; (void)e; (void)f; (void)g; misuse("synth_wah");
}
