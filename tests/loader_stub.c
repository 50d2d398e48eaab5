/* A stand-in GPU library for the loader tests (CPU only): the 15 entry points
 * of ddscat_matvec_cuda.h as no-op stubs returning 0.  Compiling with
 * -DOMIT_<NAME> leaves entry point <NAME> out, to check how the reference's
 * loader (ddscat_cuda_unified/cuda/ddscat_cuda_loader.c:41-80) reacts to a
 * missing symbol: 1000 + 2 for a mandatory one, -777 for
 * ddscat_cuda_prepare_green_f32 (:88). */
#include <stdint.h>

#define STUB(name, ...) __attribute__((visibility("default"))) int name(__VA_ARGS__) { return 0; }

#ifndef OMIT_PREPARE
STUB(ddscat_cuda_prepare_f32, int a, int b, int c, int d, int e, int f, const void* g, const int16_t* h)
#endif
#ifndef OMIT_PREPARE_GREEN
STUB(ddscat_cuda_prepare_green_f32, int a, int b, int c, int d, int e, int f, int g, float h, float i, float j,
     float k, float l, float m, float n, float o, float p, const int16_t* q)
#endif
#ifndef OMIT_APPLY
STUB(ddscat_cuda_apply_f32, int a, const void* b, void* c, const void* d, const void* e)
#endif
#define SOLVER(name) STUB(name, const void* b, void* x, const void* ad, const void* ao, int n, int m, float t, \
                          int* it, float* to, int* nc)
SOLVER(ddscat_cuda_solve_gpbicg_f32)
#ifndef OMIT_QMRCCG
SOLVER(ddscat_cuda_solve_qmrccg_f32)
#endif
SOLVER(ddscat_cuda_solve_pbcgst_f32)
SOLVER(ddscat_cuda_solve_pbcgs2_f32)
SOLVER(ddscat_cuda_solve_petrkp_f32)
SOLVER(ddscat_cuda_solve_bicgstab4_f32)
SOLVER(ddscat_cuda_solve_gpbicgstab2_f32)
SOLVER(ddscat_cuda_solve_gpbicgstab4_f32)
STUB(ddscat_cuda_evalq_f32, int a, const void* b, const void* c, const void* d, const void* e, float f, float g,
     float h, float i, double* j, double* k, double* l)
#ifndef OMIT_SCAT
STUB(ddscat_cuda_scat_f32, int a, int b, const float* c, const float* d, const float* e, const float* f,
     const float* g, float h, float i, const void* j, const float* k, double* l, double* m, double* n, double* o,
     int* p, void* q, void* r)
#endif
STUB(ddscat_cuda_release, void)
__attribute__((visibility("default"))) const char* ddscat_cuda_last_error(void) { return "stub"; }
