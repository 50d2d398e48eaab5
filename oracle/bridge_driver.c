/* Stand-in for DDSCAT's Fortran bridge (test infrastructure, not product).
 *
 * DDSCAT reaches the GPU library only through the reference's C loader
 * (ddscat_cuda_unified/cuda/ddscat_cuda_loader.c: dlopen of DDSCAT_CUDA_DLL,
 * dlsym of the 15 entry points, 1000+r on a load failure, -777 when
 * ddscat_cuda_prepare_green_f32 is absent) and the Fortran module
 * ddscat_cuda_unified/fortran/cuda_matvec_bridge.f90, which calls the
 * loader's ddscat_cuda_loader_* wrappers in this order:
 * ensure_prepared (prepare_green, :141-166) -> one solver (:200-260) ->
 * CUDA_EVALQ_GPU (:265-285, resident solution) -> CUDA_SCAT_GPU (:287-306) ->
 * CUDA_MATVEC_RELEASE (:308-310), stopping at the first nonzero status.
 * gfortran is not available here, so this C program makes the same calls
 * through the same (unmodified, separately compiled) loader.  oracle/Makefile
 * links the two into oracle/_ref/ddscat_bridge_driver.
 *
 *   ddscat_bridge_driver probe             one prepare_green call on a 2x2x2
 *                                          grid; prints the loader's status
 *   ddscat_bridge_driver run IN OUT        the bridge sequence on the inputs
 *                                          in IN, results written to OUT
 *
 * IN (little-endian, packed): int32 nx, ny, nz, ipbc, nat, nat0, idipint,
 * solver (0 gpbicg, 1 qmrccg, 2 pbcgst, 3 pbcgs2, 4 petrkp, 5 bicgstab4,
 * 6 gpbicgstab2, 7 gpbicgstab4), maxit, ndir; float32 gamma, pyd, pzd, ak[3],
 * dx[3], tol, etasca, e02, x0[3]; int16 iocc[nat]; complex64 b, adia,
 * aoff [3*nat each]; complex64 e01[3]; float32 aks, em1, em2 [3*ndir each].
 * OUT: int32 rc_prepare, rc_solve, rc_evalq, rc_scat, rc_release, itno,
 * ncompte, navg; float32 tole; float64 cabs, cext, cpha, cbksca, csca,
 * cscag[3], cscag2; complex64 x[3*nat], f1[ndir], f2[ndir].
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef int (*solver_fn)(const void*, void*, const void*, const void*, int, int, float, int*, float*, int*);

int ddscat_cuda_loader_prepare_green_f32(int, int, int, int, int, int, int, float, float, float, float, float, float,
                                         float, float, float, const int16_t*);
int ddscat_cuda_loader_solve_gpbicg_f32(const void*, void*, const void*, const void*, int, int, float, int*, float*,
                                        int*);
int ddscat_cuda_loader_solve_qmrccg_f32(const void*, void*, const void*, const void*, int, int, float, int*, float*,
                                        int*);
int ddscat_cuda_loader_solve_pbcgst_f32(const void*, void*, const void*, const void*, int, int, float, int*, float*,
                                        int*);
int ddscat_cuda_loader_solve_pbcgs2_f32(const void*, void*, const void*, const void*, int, int, float, int*, float*,
                                        int*);
int ddscat_cuda_loader_solve_petrkp_f32(const void*, void*, const void*, const void*, int, int, float, int*, float*,
                                        int*);
int ddscat_cuda_loader_solve_bicgstab4_f32(const void*, void*, const void*, const void*, int, int, float, int*, float*,
                                           int*);
int ddscat_cuda_loader_solve_gpbicgstab2_f32(const void*, void*, const void*, const void*, int, int, float, int*,
                                             float*, int*);
int ddscat_cuda_loader_solve_gpbicgstab4_f32(const void*, void*, const void*, const void*, int, int, float, int*,
                                             float*, int*);
int ddscat_cuda_loader_evalq_f32(int, const void*, const void*, const void*, const void*, float, float, float, float,
                                 double*, double*, double*);
int ddscat_cuda_loader_scat_f32(int, int, const float*, const float*, const float*, const float*, const float*, float,
                                float, const void*, const float*, double*, double*, double*, double*, int*, void*,
                                void*);
int ddscat_cuda_loader_release(void);
const char* ddscat_cuda_loader_last_error(void);

static void* slurp(FILE* f, size_t bytes) {
  void* p = malloc(bytes ? bytes : 1);
  if (!p || fread(p, 1, bytes, f) != bytes) {
    fprintf(stderr, "bridge_driver: short input\n");
    exit(2);
  }
  return p;
}

static int probe(void) {
  int16_t occ[8] = {1, 1, 1, 1, 1, 1, 1, 1};
  const int rc = ddscat_cuda_loader_prepare_green_f32(2, 2, 2, 0, 8, 8, 0, 0.f, 0.f, 0.f, 0.3f, 0.f, 0.f, 1.f, 1.f,
                                                      1.f, occ);
  printf("%d\n", rc);
  if (rc == 0) ddscat_cuda_loader_release();
  return 0;
}

static int run(const char* in_path, const char* out_path) {
  FILE* f = fopen(in_path, "rb");
  if (!f) { perror(in_path); return 2; }
  int32_t hi[10];
  float hf[15];
  if (fread(hi, sizeof(int32_t), 10, f) != 10 || fread(hf, sizeof(float), 15, f) != 15) {
    fprintf(stderr, "bridge_driver: short header\n");
    return 2;
  }
  const int nx = hi[0], ny = hi[1], nz = hi[2], ipbc = hi[3], nat = hi[4], nat0 = hi[5], idipint = hi[6];
  const int solver = hi[7], maxit = hi[8], ndir = hi[9];
  const float gamma = hf[0], pyd = hf[1], pzd = hf[2], tol = hf[9], etasca = hf[10], e02 = hf[11];
  const float* ak = hf + 3;
  const float* dx = hf + 6;
  const float* x0 = hf + 12;
  const size_t n3 = (size_t)3 * nat, cb = 2 * sizeof(float);
  int16_t* iocc = (int16_t*)slurp(f, (size_t)nat * sizeof(int16_t));
  void* b = slurp(f, n3 * cb);
  void* adia = slurp(f, n3 * cb);
  void* aoff = slurp(f, n3 * cb);
  void* e01 = slurp(f, 3 * cb);
  float* aks = (float*)slurp(f, (size_t)3 * ndir * sizeof(float));
  float* em1 = (float*)slurp(f, (size_t)3 * ndir * sizeof(float));
  float* em2 = (float*)slurp(f, (size_t)3 * ndir * sizeof(float));
  fclose(f);
  void* x = calloc(n3, cb);
  void* f1 = calloc(ndir ? ndir : 1, cb);
  void* f2 = calloc(ndir ? ndir : 1, cb);
  int32_t rcs[5] = {-1, -1, -1, -1, -1};
  int32_t itno = 0, ncompte = 0, navg = 0;
  float tole = 0.f;
  double q[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  static const solver_fn solvers[8] = {
      ddscat_cuda_loader_solve_gpbicg_f32,     ddscat_cuda_loader_solve_qmrccg_f32,
      ddscat_cuda_loader_solve_pbcgst_f32,     ddscat_cuda_loader_solve_pbcgs2_f32,
      ddscat_cuda_loader_solve_petrkp_f32,     ddscat_cuda_loader_solve_bicgstab4_f32,
      ddscat_cuda_loader_solve_gpbicgstab2_f32, ddscat_cuda_loader_solve_gpbicgstab4_f32};
  if (solver < 0 || solver > 7) { fprintf(stderr, "bridge_driver: solver id %d\n", solver); return 2; }
  /* ensure_prepared */
  rcs[0] = ddscat_cuda_loader_prepare_green_f32(nx, ny, nz, ipbc, nat, nat0, idipint, gamma, pyd, pzd, ak[0], ak[1],
                                                ak[2], dx[0], dx[1], dx[2], iocc);
  if (rcs[0] == 0) {
    /* CUDA_<solver>_SOLVE */
    int it = 0, nc = 0;
    rcs[1] = solvers[solver](b, x, adia, aoff, (int)n3, maxit, tol, &it, &tole, &nc);
    itno = it;
    ncompte = nc;
  }
  if (rcs[1] == 0) /* CUDA_EVALQ_GPU with the resident solution */
    rcs[2] = ddscat_cuda_loader_evalq_f32(1, NULL, NULL, NULL, NULL, ak[0], ak[1], ak[2], e02, &q[0], &q[1], &q[2]);
  if (rcs[2] == 0) { /* CUDA_SCAT_GPU */
    int nv = 0;
    rcs[3] = ddscat_cuda_loader_scat_f32(0, ndir, ak, aks, dx, em1, em2, e02, etasca, e01, x0, &q[3], &q[4], &q[5],
                                         &q[8], &nv, f1, f2);
    navg = nv;
  }
  rcs[4] = ddscat_cuda_loader_release(); /* CUDA_MATVEC_RELEASE */
  for (int i = 0; i < 4; ++i)
    if (rcs[i] != 0 && rcs[i] != -1) fprintf(stderr, "bridge_driver: stage %d status %d: %s\n", i, rcs[i],
                                             ddscat_cuda_loader_last_error());
  FILE* o = fopen(out_path, "wb");
  if (!o) { perror(out_path); return 2; }
  const int32_t ints[8] = {rcs[0], rcs[1], rcs[2], rcs[3], rcs[4], itno, ncompte, navg};
  fwrite(ints, sizeof(int32_t), 8, o);
  fwrite(&tole, sizeof(float), 1, o);
  fwrite(q, sizeof(double), 9, o);
  fwrite(x, cb, n3, o);
  fwrite(f1, cb, (size_t)ndir, o);
  fwrite(f2, cb, (size_t)ndir, o);
  fclose(o);
  free(iocc); free(b); free(adia); free(aoff); free(e01); free(aks); free(em1); free(em2);
  free(x); free(f1); free(f2);
  return 0;
}

int main(int argc, char** argv) {
  if (argc == 2 && strcmp(argv[1], "probe") == 0) return probe();
  if (argc == 4 && strcmp(argv[1], "run") == 0) return run(argv[2], argv[3]);
  fprintf(stderr, "usage: %s probe | run IN OUT\n", argv[0]);
  return 2;
}
